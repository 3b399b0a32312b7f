/*
 * wavefront.cuh -- the wavefront form of render.zig's per-pixel estimator.
 *
 * One path slot per pixel in flight.  Each iteration runs three kernels over
 * compacted queues of slot indices:
 *   extend  closest-hit query of every active ray          (scene.zig:108-116)
 *   shade   emission + MIS, light sample, scatter, roulette (render.zig:73-99)
 *   shadow  any-hit query of the light samples              (render.zig:50-51)
 * and a one-thread advance kernel that swaps the queues and sets the
 * condition of the CUDA-graph while node that drives the loop on the device.
 *
 * Exactness: a slot replays traceWith's operations for its pixel in the
 * reference order.  The RNG is only drawn in shade and in camera-ray
 * generation, in the reference order; the NEE term of bounce k is added to
 * the slot's radiance by the shadow kernel, which runs after shade(k) and
 * before shade(k+1), so the f64 sum radiance = ((le_0 + nee_0) + le_1) + ...
 * keeps the reference's association.  A path that ends with a light sample
 * pending is finished by the shadow kernel after the add.
 */
#ifndef ZT_WAVEFRONT_CUH
#define ZT_WAVEFRONT_CUH

#include "zt_device.cuh"

namespace zt {

/* Structure-of-arrays path state; every array has `capacity` entries. */
struct WfState {
  uint32_t* pix;      /* pixel of the slot */
  uint32_t* sample;   /* sample index within the pixel */
  uint32_t* depth;    /* bounce index of the current ray */
  uint32_t* flags;    /* bit 0: path ends after the pending shadow test */
  uint64_t* rng;      /* 4 words per slot, word-major: rng[w * cap + s] */
  double* ray;        /* o.xyz, d.xyz: 6 per slot, component-major */
  double* tp;         /* throughput */
  double* rad;        /* radiance of the current sample */
  double* sum;        /* pixel accumulator */
  double* prev;       /* prev_origin.xyz, prev_pdf */
  double* hit_t;
  int32_t* hit_k;     /* >= 0 prim, <= -2 plane (-2 - i), -1 miss */
  double* nee;        /* shadow ray o.xyz d.xyz tmax, contribution.xyz, throughput.xyz: 13 per slot */
  uint32_t* queue[2]; /* ping-pong extension queues */
  uint32_t* shadow_q; /* slots with a pending light sample */
  uint32_t* ctl;      /* [0] iter, [1] n_ext[0], [2] n_ext[1], [3] n_shadow, [4] next pixel, [5] error, [6] go */
  uint32_t* sort_key; /* queue sort: bucket of each queue entry */
  uint32_t* sort_tmp; /* queue sort: the sorted queue before it is copied back */
  uint32_t* sort_hist;/* queue sort: kSortBuckets counts, then running offsets */
  uint32_t capacity;
};

enum { kCtlIter = 0, kCtlExt0 = 1, kCtlShadow = 3, kCtlNextPixel = 4, kCtlError = 5, kCtlGo = 6 };

/* Extension rays are sorted between iterations by direction octant (3 bits)
 * and the cell of their origin on an 8x8x8 grid over the scene bounds
 * (9 bits, Morton order): rays in one warp then start near one another and
 * head the same way, so they walk more of the same BVH nodes together. */
constexpr uint32_t kSortCellBits = 3;
constexpr uint32_t kSortBuckets = 8u << (3 * kSortCellBits);

ZT_D dv3 ld3(const double* a, uint32_t cap, uint32_t s, int c0) {
  return V(a[(size_t)c0 * cap + s], a[(size_t)(c0 + 1) * cap + s], a[(size_t)(c0 + 2) * cap + s]);
}
ZT_D void st3(double* a, uint32_t cap, uint32_t s, int c0, dv3 v) {
  a[(size_t)c0 * cap + s] = v.x;
  a[(size_t)(c0 + 1) * cap + s] = v.y;
  a[(size_t)(c0 + 2) * cap + s] = v.z;
}
ZT_D Rng ld_rng(const WfState& w, uint32_t s) {
  const size_t c = w.capacity;
  return Rng{w.rng[s], w.rng[c + s], w.rng[2 * c + s], w.rng[3 * c + s]};
}
ZT_D void st_rng(const WfState& w, uint32_t s, const Rng& r) {
  const size_t c = w.capacity;
  w.rng[s] = r.s0;
  w.rng[c + s] = r.s1;
  w.rng[2 * c + s] = r.s2;
  w.rng[3 * c + s] = r.s3;
}

/* Warp-aggregated append of slot s to queue q with counter *n. */
ZT_D void push(uint32_t* q, uint32_t* n, uint32_t s) {
  const unsigned mask = __activemask();
  const int leader = __ffs(mask) - 1;
  const unsigned lane = threadIdx.x & 31;
  uint32_t base = 0;
  if ((int)lane == leader) base = atomicAdd(n, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  q[base + __popc(mask & ((1u << lane) - 1))] = s;
}

/* Camera ray of the slot's current sample (render.zig:138-140). */
ZT_D void start_sample(const WfState& w, const RenderParams& p, uint32_t s, Rng& rng) {
  const uint64_t pix = w.pix[s];
  const uint64_t x = pix % p.width, y = pix / p.width;
  const double sx = ((double)x + rng_float(rng)) / (double)p.width;
  const double ty = ((double)y + rng_float(rng)) / (double)p.height;
  dv3 ro, rd;
  camera_ray(p.cam, sx, ty, rng, ro, rd);
  const uint32_t c = w.capacity;
  st3(w.ray, c, s, 0, ro);
  st3(w.ray, c, s, 3, rd);
  st3(w.tp, c, s, 0, V(1, 1, 1));
  st3(w.rad, c, s, 0, V(0, 0, 0));
  st3(w.prev, c, s, 0, V(0, 0, 0));
  w.prev[3 * (size_t)c + s] = 0.0;
  w.depth[s] = 0;
  w.flags[s] = 0;
}

/* Starts pixel `pix` in slot s (render.zig:135-136). */
ZT_D void start_pixel(const WfState& w, const RenderParams& p, uint32_t s, uint32_t pix, Rng& rng) {
  w.pix[s] = pix;
  w.sample[s] = 0;
  st3(w.sum, w.capacity, s, 0, V(0, 0, 0));
  rng = rng_for_stream(p.seed, pix);
}

/* End of a sample: accumulate (render.zig:141-142), then the next sample of
 * the pixel, or write the pixel and take a new one.  Pushes the slot's next
 * ray to `q`. */
ZT_D void finish_sample(const WfState& w, const RenderParams& p, uint32_t s, Rng& rng, double* __restrict__ out,
                        uint32_t* q, uint32_t* n) {
  const uint32_t c = w.capacity;
  const dv3 r = ld3(w.rad, c, s, 0);
  dv3 sum = ld3(w.sum, c, s, 0);
  if (visfinite(r)) sum = sum + r;
  const uint32_t next = w.sample[s] + 1;
  if (next < p.spp) {
    st3(w.sum, c, s, 0, sum);
    w.sample[s] = next;
    start_sample(w, p, s, rng);
    st_rng(w, s, rng);
    push(q, n, s);
    return;
  }
  const dv3 px = vscale(sum, 1.0 / (double)p.spp); /* render.zig:144 */
  const uint64_t pix = w.pix[s];
  out[3 * pix + 0] = px.x;
  out[3 * pix + 1] = px.y;
  out[3 * pix + 2] = px.z;
  const uint32_t np = atomicAdd(&w.ctl[kCtlNextPixel], 1u);
  if ((uint64_t)np < p.width * p.height) {
    start_pixel(w, p, s, np, rng);
    start_sample(w, p, s, rng);
    st_rng(w, s, rng);
    push(q, n, s);
  }
}

}  // namespace zt

#endif

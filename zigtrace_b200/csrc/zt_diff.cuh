/*
 * zt_diff.cuh -- the differentiable form of traceWith: gradients of an image
 * loss with respect to every material's colour (the albedo of Lambertian and
 * metal materials, the radiance of emissive ones).
 *
 * Detached sampling.  The scene's own materials (theta0) drive every sampling
 * decision: the roulette probability comes from a throughput built with
 * theta0's albedos, the light pick from the theta0 emitter table, and the MIS
 * weights from theta0's pdfs.  Contributions are evaluated with the parameters
 * theta.  Each sample is then a product of parameter factors times constants
 * fixed by the random numbers, so with common random numbers it is a smooth
 * function of theta, and its expectation is the rendering at theta (an
 * importance-sampled estimator with a fixed proposal is unbiased).  At
 * theta == theta0 every operation is traceWith's (render.zig:61-102) in the
 * same order, so the image is the reference image bit for bit.
 *
 * Path replay.  The adjoint of one sample re-runs its path from the saved RNG
 * state (no tape).  A scatter at material m multiplies every term added
 * after it by theta[m], so d/d theta[m] gets adj * (L - R) / theta[m], with L
 * the sample's radiance (from the primal pass) and R the radiance added so
 * far; emission and light-sample terms add their own direct derivatives.
 * A zero albedo channel contributes no gradient (the proposal never
 * continues a path past it).
 */
#ifndef ZT_DIFF_CUH
#define ZT_DIFF_CUH

#include "zt_device.cuh"

namespace zt {

/* Adds v to grad[3m..3m+2].  warp_private: grad is this warp's own slice of
 * shared memory, so the active lanes add in turn with plain loads and
 * stores (no atomics, no contention with other warps); otherwise global
 * atomics. */
ZT_D void grad_add(double* grad, bool warp_private, uint32_t m, dv3 v) {
  double* q = grad + 3 * (size_t)m;
  if (!warp_private) {
    atomicAdd(q + 0, v.x);
    atomicAdd(q + 1, v.y);
    atomicAdd(q + 2, v.z);
    return;
  }
  const unsigned mask = __activemask();
  const int lane = (int)(threadIdx.x & 31);
  for (unsigned mk = mask; mk; mk &= mk - 1) {
    if (lane == __ffs(mk) - 1) {
      q[0] += v.x;
      q[1] += v.y;
      q[2] += v.z;
    }
    __syncwarp(mask);
  }
}

/* The BVH query as a real call: the differentiable kernels are instruction-
 * cache bound when each of their queries inlines its own copy of the
 * traversal (measured: forward and backward ~22% faster outlined). */
__device__ __noinline__ int32_t scene_query_outlined(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax,
                                                     bool any_hit, double& t_out) {
  return scene_query_rt(sc, o, d, tmin, tmax, any_hit, t_out);
}

/* kAdj is a run-time flag so that the primal and the replay pass of the
 * backward kernel share one copy of this code (the kernel is instruction-
 * cache bound with two copies). */
ZT_D dv3 trace_diff(const DevScene& sc, const double* __restrict__ theta, dv3 ro, dv3 rd, Rng& rng,
                    uint64_t max_depth, bool use_nee, bool kAdj, dv3 L_total, dv3 adj, double* grad,
                    bool warp_private) {
  dv3 radiance = V(0, 0, 0), tp = V(1, 1, 1), tp0 = V(1, 1, 1);
  /* prev_origin (render.zig:66-70) is read only after a bounce, where it
   * equals ro: ro stands in for it, as in trace_with */
  double prev_pdf = 0;
  for (uint64_t depth = 0; depth < max_depth; ++depth) {
    Hit hit;
    double th_t;
    const int32_t hk = scene_query_outlined(sc, ro, rd, kRayEpsilon, INFINITY, false, th_t);
    if (hk == -1) return radiance + vmul(tp, background_radiance(sc.bg, rd));
    hit_from(sc, hk, ro, rd, th_t, hit);
    const uint32_t m = hit.material;
    const DMat& mat = sc.mats[m];
    const dv3 th = L3(theta + 3 * (size_t)m);
    const bool emits = mat.kind == kEmissive && hit.front_face;
    const dv3 le0 = emits ? L3(mat.color) : V(0, 0, 0);
    if (vmaxc(le0) > 0) { /* emission with its MIS weight, render.zig:77-81 */
      const double w = prev_pdf > 0 ? power_weight(prev_pdf, lights_pdf_hit(sc, ro, hit.point)) : 1.0;
      if (kAdj) grad_add(grad, warp_private, m, vmul(adj, vscale(tp, w)));
      radiance = radiance + vscale(vmul(tp, th), w);
    }
    if (mat.kind == kLambertian && use_nee) { /* directLight, render.zig:46-56 */
      dv3 ldir, lrad0, direct = V(0, 0, 0);
      double ldist, lpdf;
      uint32_t li = 0;
      if (lights_sample(sc, hit.point, rng, ldir, ldist, lrad0, lpdf, &li)) {
        const double cos_s = vdot(hit.normal, ldir);
        if (!(cos_s <= 0 || !(lpdf > 0))) {
          double st;
          if (scene_query_outlined(sc, hit.point, ldir, kRayEpsilon, ldist * (1 - 1e-6), true, st) == -1) {
            const double bsdf_pdf = cos_s / kPi;
            const double scale = cos_s / (kPi * lpdf) * power_weight(lpdf, bsdf_pdf);
            const uint32_t lm = sc.lights[li].material;
            const dv3 lrad = L3(theta + 3 * (size_t)lm);
            direct = vscale(vmul(th, lrad), scale);
            if (kAdj) {
              grad_add(grad, warp_private, m, vmul(adj, vscale(vmul(tp, lrad), scale)));
              grad_add(grad, warp_private, lm, vmul(adj, vscale(vmul(tp, th), scale)));
            }
          }
        }
      }
      radiance = radiance + vmul(tp, direct);
    }
    dv3 atten0, sd;
    if (!material_scatter(mat, rd, hit, rng, atten0, sd)) break;
    const bool param = mat.kind == kLambertian || mat.kind == kMetal;
    const dv3 atten = param ? th : atten0;
    if (kAdj && param) { /* every later term carries atten: their sum is L_total - radiance */
      const dv3 rest = L_total - radiance;
      grad_add(grad, warp_private, m, V(atten.x != 0 ? adj.x * rest.x / atten.x : 0.0, atten.y != 0 ? adj.y * rest.y / atten.y : 0.0,
                          atten.z != 0 ? adj.z * rest.z / atten.z : 0.0));
    }
    tp = vmul(tp, atten);
    tp0 = vmul(tp0, atten0);
    prev_pdf = (use_nee && mat.kind == kLambertian) ? fmax(vdot(sd, hit.normal), 0.0) / kPi : 0;
    ro = hit.point;
    rd = sd;
    if (depth + 1 >= kRouletteDepth) { /* roulette on the theta0 throughput */
      const double p = fmin(vmaxc(tp0), 0.95);
      if (p <= 0 || rng_float(rng) >= p) break;
      tp = vdiv(tp, p);
      tp0 = vdiv(tp0, p);
    }
  }
  return radiance;
}

}  // namespace zt

#endif

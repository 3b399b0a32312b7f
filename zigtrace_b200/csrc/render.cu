/*
 * render.cu -- device residency, the radiance kernels and the render entry
 * points of the C ABI (include/zigtrace_b200.h).
 *
 * Work decomposition: render.zig:104-180 hands 16x16 tiles to host threads
 * from an atomic counter, and each pixel draws its samples from one
 * xoshiro256++ stream seeded by (seed, pixel index) (render.zig:135).  The
 * samples of a pixel are therefore sequential; pixels are independent.  The
 * megakernel runs one pixel per thread, all of its samples in order, with a
 * persistent grid that takes pixel batches from a device work counter.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "scene_host.h"
#include "output.cuh"
#include "wavefront.cuh"
#include "zt_device.cuh"
#include "zt_diff.cuh"

using namespace zt;

/* Pinned host image of the flattened scene: every device array at a 256-byte
 * aligned offset in one block, so an upload is a single host-to-device copy
 * from pinned memory into a single device allocation. */
struct zt_host_staging {
  void* pinned = nullptr;
  size_t bytes = 0;
  size_t off_prims = 0, off_ids = 0, off_pairs = 0, off_fpairs = 0, off_planes = 0, off_mats = 0, off_lights = 0,
         off_cdf = 0;
  DevScene view;  /* counts, root, total; pointers unset */
};

/* Wavefront path state (grow-only) and the cached executable graph that
 * drives it.  The graph bakes its kernel arguments in, so it is reused only
 * for an identical launch (same scene view, parameters and output). */
struct zt_wavefront_cache {
  void* block = nullptr;
  size_t bytes = 0;
  uint32_t capacity = 0;
  zt::WfState state;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;  /* recorded after the last launch of exec */
  unsigned char key[sizeof(zt::DevScene) + sizeof(zt::RenderParams) + sizeof(void*) + 2 * sizeof(uint64_t)] = {};
};

/* The per-sample primal radiance of the last zt_forward, with everything it
 * depends on: options, parameters, camera and background.  A zt_backward
 * with the same ones replays paths against it instead of recomputing the
 * primal; any difference (another view rendered in between, for instance)
 * makes the backward recompute. */
struct zt_diff_cache {
  double* L = nullptr;
  size_t cap = 0; /* doubles */
  bool valid = false;
  zt_options opts{};
  uint64_t row0 = 0, rows = 0; /* the band the cached samples belong to */
  std::vector<double> theta;
  zt_camera_config camera{};
  zt_background background{};
};

struct zt_device_buffers {
  int device = -1;
  void* block = nullptr;           /* all scene arrays */
  unsigned int* counter = nullptr; /* work counter of the persistent grid */
  DevScene view;
  zt_wavefront_cache wf;
  zt_diff_cache diff;
};

namespace zt {

static zt_status cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? ZT_ERR_OUT_OF_MEMORY : ZT_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}

#define ZT_CUDA(call, what)                       \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

/* Stream-ordered allocations from one memory pool per device, for the
 * buffers the synchronous entry points need per call or per upload (the
 * scene block, framebuffers).  Memory freed into the pool stays reserved
 * for the next allocation, up to kPoolKeepBytes across synchronisations, so
 * re-uploading a scene or rendering into host buffers frame after frame
 * costs no cudaMalloc/cudaFree pair (each maps or unmaps device pages and
 * synchronises the device). */
constexpr uint64_t kPoolKeepBytes = 4ull << 30;
static std::mutex g_pool_mutex;
static cudaMemPool_t g_pools[256] = {};

static zt_status device_pool(cudaMemPool_t* out) {
  int dev = 0;
  ZT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= 256) return fail(ZT_ERR_INVALID_ARGUMENT, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (!g_pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof props);
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    ZT_CUDA(cudaMemPoolCreate(&pool, &props), "cudaMemPoolCreate");
    uint64_t keep = kPoolKeepBytes;
    ZT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    g_pools[dev] = pool;
  }
  *out = g_pools[dev];
  return ZT_OK;
}

static zt_status pool_alloc(void** p, size_t bytes, cudaStream_t st, const char* what) {
  cudaMemPool_t pool = nullptr;
  zt_status rc = device_pool(&pool);
  if (rc != ZT_OK) return rc;
  ZT_CUDA(cudaMallocFromPoolAsync(p, bytes > 0 ? bytes : 256, pool, st), what);
  return ZT_OK;
}

static void pool_free(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

void release_device(zt_scene* s) {
  zt_device_buffers* d = s->device;
  if (!d) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (d->device >= 0 && d->device != cur) cudaSetDevice(d->device);
  /* work on any stream may still read the scene: wait for it, as cudaFree would */
  cudaDeviceSynchronize();
  if (d->wf.exec) cudaGraphExecDestroy(d->wf.exec);
  if (d->wf.done) cudaEventDestroy(d->wf.done);
  cudaFree(d->wf.block);
  cudaFree(d->diff.L);
  pool_free(d->block, 0);
  pool_free(d->counter, 0);
  cudaStreamSynchronize(0);
  if (d->device >= 0 && d->device != cur) cudaSetDevice(cur);
  delete d;
  s->device = nullptr;
}

void release_staging(zt_scene* s) {
  release_device(s);
  if (!s->staging) return;
  cudaFreeHost(s->staging->pinned);
  delete s->staging;
  s->staging = nullptr;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

template <typename T>
static void stage(const std::vector<T>& v, size_t& cursor, size_t& off) {
  off = cursor;
  cursor = align256(cursor + v.size() * sizeof(T));
}

template <typename T>
static void stage_copy(const std::vector<T>& v, void* base, size_t off) {
  if (!v.empty()) memcpy((char*)base + off, v.data(), v.size() * sizeof(T));
}

/* Flattens the built scene into one pinned block (once per build). */
static zt_status make_staging(zt_scene* s) {
  if (s->staging) return ZT_OK;
  FlatScene f;
  try {
    flatten_scene(s, &f);
  } catch (const std::bad_alloc&) {
    return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory while flattening the scene");
  }
  zt_host_staging* h = new (std::nothrow) zt_host_staging();
  if (!h) return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory");
  size_t cur = 0;
  stage(f.prims, cur, h->off_prims);
  stage(f.prim_ids, cur, h->off_ids);
  stage(f.pairs, cur, h->off_pairs);
  stage(f.fpairs, cur, h->off_fpairs);
  stage(f.planes, cur, h->off_planes);
  stage(f.mats, cur, h->off_mats);
  stage(f.lights, cur, h->off_lights);
  stage(f.cdf, cur, h->off_cdf);
  h->bytes = cur > 0 ? cur : 256;
  cudaError_t e = cudaMallocHost(&h->pinned, h->bytes);
  if (e != cudaSuccess) {
    delete h;
    return cuda_fail(e, "allocate pinned staging");
  }
  memset(h->pinned, 0, h->bytes);
  stage_copy(f.prims, h->pinned, h->off_prims);
  stage_copy(f.prim_ids, h->pinned, h->off_ids);
  stage_copy(f.pairs, h->pinned, h->off_pairs);
  stage_copy(f.fpairs, h->pinned, h->off_fpairs);
  stage_copy(f.planes, h->pinned, h->off_planes);
  stage_copy(f.mats, h->pinned, h->off_mats);
  stage_copy(f.lights, h->pinned, h->off_lights);
  stage_copy(f.cdf, h->pinned, h->off_cdf);
  h->view = f.view;
  s->staging = h;
  return ZT_OK;
}

static zt_status pilot_paths(zt_scene* s);

/* Makes the scene resident on the current device.  With sync = false the
 * host-to-device copy is left in flight on the legacy default stream (work
 * later enqueued there, or after a synchronisation, sees it): a caller
 * uploading many scenes synchronises once. */
static zt_status upload(zt_scene* s, bool sync = true) {
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built: call zt_scene_build first");
  int dev = 0;
  ZT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (s->device && s->device->device == dev) return s->pilot_valid ? ZT_OK : pilot_paths(s);
  release_device(s);
  zt_status rc = make_staging(s);
  if (rc != ZT_OK) return rc;
  const zt_host_staging* h = s->staging;
  zt_device_buffers* d = new (std::nothrow) zt_device_buffers();
  if (!d) return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory");
  d->device = dev;
  s->device = d;
  zt_status arc = pool_alloc(&d->block, h->bytes, 0, "allocate the scene block");
  if (arc == ZT_OK) arc = pool_alloc((void**)&d->counter, 4 * sizeof(unsigned int), 0, "allocate the work counter");
  if (arc != ZT_OK) {
    release_device(s);
    return arc;
  }
  cudaError_t e = cudaMemcpyAsync(d->block, h->pinned, h->bytes, cudaMemcpyHostToDevice, 0);
  if (e == cudaSuccess && sync) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) {
    release_device(s);
    return cuda_fail(e, "upload scene");
  }
  char* b = (char*)d->block;
  d->view = h->view;
  d->view.prims = (const DPrim*)(b + h->off_prims);
  d->view.prim_ids = (const int32_t*)(b + h->off_ids);
  d->view.pairs = (const DPair*)(b + h->off_pairs);
  d->view.fpairs = h->view.fast_ok ? (const FPair*)(b + h->off_fpairs) : nullptr;
  d->view.planes = (const DPrim*)(b + h->off_planes);
  d->view.mats = (const DMat*)(b + h->off_mats);
  d->view.lights = (const DLight*)(b + h->off_lights);
  d->view.cdf = (const double*)(b + h->off_cdf);
  return s->pilot_valid ? ZT_OK : pilot_paths(s);
}

/* The resident view with the scene's current background (the background can
 * change after upload without touching device memory). */
static DevScene launch_view(const zt_scene* s) {
  DevScene v = s->device->view;
  const zt_background& bg = s->background;
  v.bg.kind = bg.kind;
  v.bg.a[0] = bg.a.x; v.bg.a[1] = bg.a.y; v.bg.a[2] = bg.a.z;
  v.bg.b[0] = bg.b.x; v.bg.b[1] = bg.b.y; v.bg.b[2] = bg.b.z;
  return v;
}

static bool options_valid(const zt_options* o) { /* render.zig:153 */
  return !(o->width == 0 || o->height == 0 || o->spp == 0 || o->tile_size == 0);
}

static RenderParams make_params(const zt_scene* s, const zt_options* o) {
  RenderParams p;
  p.cam = camera_init(s->camera, (double)o->width / (double)o->height); /* render.zig:157, 162 */
  p.width = o->width;
  p.height = o->height;
  p.spp = o->spp;
  p.max_depth = o->max_depth;
  p.seed = o->seed;
  p.use_nee = (o->light_sampling && !s->lights.empty()) ? 1u : 0u; /* render.zig:62 */
  p.row0 = 0;
  p.rows = o->height;
  p.pad = 0;
  return p;
}

/* ------------------------------------------------------------ Kernels ---- */

/* One pixel: renderTile's per-pixel body, render.zig:133-144.  kNee as for
 * trace_with. */
template <bool kAux, bool kNee = true, bool kFast = false>
__device__ __forceinline__ void render_pixel(const DevScene& sc, const RenderParams& p, uint64_t pix,
                                             double* __restrict__ out, TraceAux* aux) {
  const uint64_t x = pix % p.width, y = pix / p.width;
  const double w = (double)p.width, h = (double)p.height;
  const double inv_spp = 1.0 / (double)p.spp;
  Rng rng = rng_for_stream(p.seed, y * p.width + x);
  dv3 sum = V(0, 0, 0);
  for (uint64_t i = 0; i < p.spp; ++i) {
    const double s = ((double)x + rng_float(rng)) / w;
    const double t = ((double)y + rng_float(rng)) / h;
    dv3 ro, rd;
    camera_ray(p.cam, s, t, rng, ro, rd);
    const dv3 c = trace_with<kAux, kNee, kFast>(sc, ro, rd, rng, p.max_depth, p.use_nee != 0, aux);
    if (kAux) break;
    if (visfinite(c)) sum = sum + c;
  }
  if (!kAux) {
    const dv3 px = vscale(sum, inv_spp);
    const uint64_t o = pix - p.row0 * p.width; /* output starts at the band's first row */
    out[3 * o + 0] = px.x;
    out[3 * o + 1] = px.y;
    out[3 * o + 2] = px.z;
  }
}

/* Persistent megakernel: each warp takes an 8x4 pixel tile from the device
 * work counter until the image is exhausted (the device form of
 * Context.work's atomic tile counter, render.zig:113-119), so its camera rays
 * are coherent.  The exact instance with light sampling is built for 1024
 * resident threads per SM (64 registers): on the 1M-triangle terrain 731
 * Msamples/s against 722 at 896 (an earlier source measured 896 fastest).
 * The instance without light sampling (kNee = false) is a separate build
 * with its own residency: 896 threads (72 registers), equal to 1024 on the
 * random spheres (2798 against 2794). */
constexpr int kMegaThreadsPerSm = 1024;
constexpr int kMegaThreadsPerSmNoNee = 896;
#ifndef ZT_FAST_THREADS_PER_SM
#define ZT_FAST_THREADS_PER_SM 1024
#endif
#ifndef ZT_FAST_THREADS_PER_SM_NONEE
#define ZT_FAST_THREADS_PER_SM_NONEE 1024
#endif
/* Resident threads per SM each megakernel and batch instance is built for
 * (__launch_bounds__): sets the register budget, 65,536 / threads.  The
 * fast-walk instances measured fastest at 1024 (64 registers): on the
 * 1M-triangle terrain 1026 Msamples/s against 992 at 896 and 933 at 768; on
 * the sphere-field batch 64.4 ms against 67.9 at 896 and 71.7 at 1280. */
__host__ __device__ constexpr int mega_threads_per_sm(bool nee, bool fast) {
  return fast ? (nee ? ZT_FAST_THREADS_PER_SM : ZT_FAST_THREADS_PER_SM_NONEE)
              : (nee ? kMegaThreadsPerSm : kMegaThreadsPerSmNoNee);
}

template <int BS, bool kNee, bool kFast = false>
__global__ void __launch_bounds__(BS, mega_threads_per_sm(kNee, kFast) / BS)
    k_render_mega(DevScene sc, RenderParams p, double* __restrict__ out, unsigned int* __restrict__ counter) {
  const uint64_t tiles_x = (p.width + 7) / 8, tiles = tiles_x * ((p.rows + 3) / 4);
  const uint64_t row_end = p.row0 + p.rows;
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= tiles) return;
    const uint64_t x = (tile % tiles_x) * 8 + (lane & 7), y = p.row0 + (tile / tiles_x) * 4 + (lane >> 3);
    if (x < p.width && y < row_end) render_pixel<false, kNee, kFast>(sc, p, y * p.width + x, out, nullptr);
  }
}

/* render_pixel with per-lane path regeneration: a lane whose path ends starts
 * its pixel's next sample at once instead of waiting at the sample boundary
 * for the longest path of its warp.  Per lane the operations and RNG draws
 * are render_pixel's and trace_with's in the same order (render.zig:61-102,
 * 133-144), so the pixel is bit-identical; only the warp's schedule changes.
 * All 32 lanes of the warp must call it (lanes outside the image with
 * valid = false).  Pays off when path lengths vary widely within a warp
 * (closed scenes such as the Cornell box); on open scenes with short paths
 * the nested form is faster. */
template <bool kFast>
__device__ __forceinline__ void render_pixel_regen(const DevScene& sc, const RenderParams& p, uint64_t x, uint64_t y,
                                                   bool valid, double* __restrict__ out) {
  const double w = (double)p.width, h = (double)p.height;
  const bool use_nee = p.use_nee != 0;
  Rng rng = rng_for_stream(p.seed, valid ? y * p.width + x : 0);
  dv3 sum = V(0, 0, 0);
  uint64_t sample = 0, depth = 0;
  bool done = !valid, fresh = valid;
  /* prev_origin (render.zig:66-70) is read only after a bounce, where it
   * equals ro: ro stands in for it, as in trace_with */
  dv3 ro = V(0, 0, 0), rd = V(0, 0, 0), radiance = V(0, 0, 0), throughput = V(1, 1, 1);
  double prev_pdf = 0;
  for (;;) {
    if (fresh) { /* render.zig:138-140: the next sample's camera ray */
      fresh = false;
      if (sample == p.spp) {
        done = true;
      } else {
        const double s = ((double)x + rng_float(rng)) / w;
        const double t = ((double)y + rng_float(rng)) / h;
        camera_ray(p.cam, s, t, rng, ro, rd);
        radiance = V(0, 0, 0);
        throughput = V(1, 1, 1);
        prev_pdf = 0;
        depth = 0;
      }
    }
    if (__all_sync(0xffffffffu, done)) break;
    if (done) continue;
    /* one iteration of traceWith's bounce loop */
    bool end = depth >= p.max_depth;
    if (!end) {
      Hit hit;
      if (!scene_intersect<false, kFast>(sc, ro, rd, kRayEpsilon, INFINITY, hit)) {
        radiance = radiance + vmul(throughput, background_radiance(sc.bg, rd));
        end = true;
      } else {
        const DMat& mat = sc.mats[hit.material];
        const dv3 le = (mat.kind == kEmissive && hit.front_face) ? L3(mat.color) : V(0, 0, 0);
        if (vmaxc(le) > 0) {
          const double wt = prev_pdf > 0 ? power_weight(prev_pdf, lights_pdf_hit<kFast>(sc, ro, hit.point)) : 1.0;
          radiance = radiance + vscale(vmul(throughput, le), wt);
        }
        if (mat.kind == kLambertian && use_nee)
          radiance = radiance + vmul(throughput, direct_light<kFast>(sc, L3(mat.color), hit, rng));
        dv3 atten, sd;
        if (!material_scatter(mat, rd, hit, rng, atten, sd)) {
          end = true;
        } else {
          throughput = vmul(throughput, atten);
          prev_pdf = (use_nee && mat.kind == kLambertian) ? fmax(vdot(sd, hit.normal), 0.0) / kPi : 0;
          ro = hit.point;
          rd = sd;
          if (depth + 1 >= kRouletteDepth) {
            const double pr = fmin(vmaxc(throughput), 0.95);
            if (pr <= 0 || rng_float(rng) >= pr) end = true;
            else throughput = vdiv(throughput, pr);
          }
          depth += 1;
          if (depth >= p.max_depth) end = true;
        }
      }
    }
    if (end) { /* render.zig:141-142 */
      if (visfinite(radiance)) sum = sum + radiance;
      ++sample;
      fresh = true;
    }
  }
  if (valid) {
    const dv3 px = vscale(sum, 1.0 / (double)p.spp);
    const uint64_t o = (y - p.row0) * p.width + x;
    out[3 * o + 0] = px.x;
    out[3 * o + 1] = px.y;
    out[3 * o + 2] = px.z;
  }
}

/* The megakernel's tile loop over render_pixel_regen.  Four blocks of 128
 * per SM (up to 128 registers, no spills): 1.17x the seven-block build on the
 * Cornell box, whose 65,536 pixels fill only a quarter of the GPU's thread
 * slots anyway, and equal to it on 1280x720 random spheres. */
template <int BS, bool kFast = false>
__global__ void __launch_bounds__(BS, 512 / BS) k_render_regen(DevScene sc, RenderParams p, double* __restrict__ out,
                                                             unsigned int* __restrict__ counter) {
  const uint64_t tiles_x = (p.width + 7) / 8, tiles = tiles_x * ((p.rows + 3) / 4);
  const uint64_t row_end = p.row0 + p.rows;
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= tiles) return;
    const uint64_t x = (tile % tiles_x) * 8 + (lane & 7), y = p.row0 + (tile / tiles_x) * 4 + (lane >> 3);
    render_pixel_regen<kFast>(sc, p, x, y, x < p.width && y < row_end, out);
  }
}

/* One render of a batch: its scene view, parameters, output and the index
 * of its first tile in the batch-wide tile numbering. */
struct BatchItem {
  DevScene sc;
  RenderParams p;
  double* out;
  uint64_t tile_begin;
  uint64_t tiles_x;
};

/* Batched persistent launch: many renders of uneven size share one grid.
 * Warps take 8x4 tiles from one counter over the concatenated tile ranges of
 * all items (in the order the host chose, largest first by default) and
 * render them with the item's own scene and parameters, so small images do
 * not leave the GPU idle the way one launch per image does.  kNee = false
 * is the instance for batches in which no render samples lights. */
template <int BS, bool kNee, bool kFast = false>
__global__ void __launch_bounds__(BS, mega_threads_per_sm(kNee, kFast) / BS)
    k_render_batch(const BatchItem* __restrict__ items, uint32_t n_items, uint64_t total_tiles,
                   unsigned int* __restrict__ counter) {
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= total_tiles) return;
    uint32_t lo = 0, hi = n_items - 1; /* last item with tile_begin <= tile */
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) / 2;
      if (items[mid].tile_begin <= tile) lo = mid;
      else hi = mid - 1;
    }
    const BatchItem& it = items[lo];
    const uint64_t local = tile - it.tile_begin;
    const uint64_t x = (local % it.tiles_x) * 8 + (lane & 7), y = (local / it.tiles_x) * 4 + (lane >> 3);
    if (x < it.p.width && y < it.p.height)
      render_pixel<false, kNee, kFast>(it.sc, it.p, y * it.p.width + x, it.out, nullptr);
  }
}

/* The batched launch with per-lane path regeneration (render_pixel_regen):
 * the same tiles and items, but a lane whose path ends starts its pixel's
 * next sample at once.  Built like k_render_regen (four blocks of 128 per
 * SM, 128 registers).  Every lane of a warp calls render_pixel_regen, lanes
 * outside their image with valid = false. */
template <int BS, bool kFast>
__global__ void __launch_bounds__(BS, 512 / BS)
    k_render_batch_regen(const BatchItem* __restrict__ items, uint32_t n_items, uint64_t total_tiles,
                         unsigned int* __restrict__ counter) {
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= total_tiles) return;
    uint32_t lo = 0, hi = n_items - 1; /* last item with tile_begin <= tile */
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) / 2;
      if (items[mid].tile_begin <= tile) lo = mid;
      else hi = mid - 1;
    }
    const BatchItem& it = items[lo];
    const uint64_t local = tile - it.tile_begin;
    const uint64_t x = (local % it.tiles_x) * 8 + (lane & 7), y = (local / it.tiles_x) * 4 + (lane >> 3);
    render_pixel_regen<kFast>(it.sc, it.p, x, y, x < it.p.width && y < it.p.height, it.out);
  }
}

__global__ void k_render_debug(DevScene sc, RenderParams p, int32_t* __restrict__ first_prim,
                               uint32_t* __restrict__ path_len) {
  const uint64_t pix = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= p.width * p.height) return;
  TraceAux aux;
  render_pixel<true>(sc, p, pix, nullptr, &aux);
  first_prim[pix] = aux.first_prim;
  path_len[pix] = aux.path_len;
}

__global__ void k_rng_streams(uint64_t seed, uint64_t stream0, uint64_t n_streams, uint64_t n_draws,
                              uint64_t* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_streams) return;
  Rng r = rng_for_stream(seed, stream0 + i);
  for (uint64_t k = 0; k < n_draws; ++k) out[i * n_draws + k] = rng_next(r);
}

/* ------------------------------------------------------------ Wavefront ---- */

/* Slots 0..n0-1 start pixels 0..n0-1 (render.zig:135-140). */
__global__ void k_wf_init(RenderParams p, WfState w, uint32_t n0) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    w.ctl[kCtlIter] = 0;
    w.ctl[kCtlExt0] = n0;
    w.ctl[kCtlExt0 + 1] = 0;
    w.ctl[kCtlShadow] = 0;
    w.ctl[kCtlNextPixel] = n0;
    w.ctl[kCtlError] = 0;
  }
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n0; s += gridDim.x * blockDim.x) {
    Rng rng;
    start_pixel(w, p, s, s, rng);
    start_sample(w, p, s, rng);
    st_rng(w, s, rng);
    w.queue[0][s] = s;
  }
}

/* Closest hit of every queued ray (scene.zig:108-116). */
__global__ void __launch_bounds__(128) k_wf_extend(DevScene sc, WfState w) {
  const uint32_t cur = w.ctl[kCtlIter] & 1;
  const uint32_t n = w.ctl[kCtlExt0 + cur];
  const uint32_t* __restrict__ q = w.queue[cur];
  const uint32_t c = w.capacity;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = q[i];
    double t;
    const int32_t k = scene_query<false>(sc, ld3(w.ray, c, s, 0), ld3(w.ray, c, s, 3), kRayEpsilon, INFINITY, t);
    w.hit_t[s] = t;
    w.hit_k[s] = k;
  }
}

/* One bounce of traceWith after the intersection (render.zig:73-99); the
 * light sample's visibility is left to k_wf_shadow. */
__global__ void __launch_bounds__(128) k_wf_shade(DevScene sc, RenderParams p, WfState w, double* __restrict__ out) {
  const uint32_t it = w.ctl[kCtlIter];
  const uint32_t cur = it & 1, nxt = cur ^ 1;
  const uint32_t n = w.ctl[kCtlExt0 + cur];
  const uint32_t* __restrict__ q = w.queue[cur];
  uint32_t* qn = w.queue[nxt];
  uint32_t* nn = &w.ctl[kCtlExt0 + nxt];
  const uint32_t c = w.capacity;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = q[i];
    Rng rng = ld_rng(w, s);
    const dv3 o = ld3(w.ray, c, s, 0), d = ld3(w.ray, c, s, 3);
    dv3 tp = ld3(w.tp, c, s, 0);
    dv3 rad = ld3(w.rad, c, s, 0);
    const int32_t k = w.hit_k[s];
    if (k == -1) { /* miss: background, render.zig:73-75 */
      rad = rad + vmul(tp, background_radiance(sc.bg, d));
      st3(w.rad, c, s, 0, rad);
      finish_sample(w, p, s, rng, out, qn, nn);
      continue;
    }
    Hit hit;
    hit_from(sc, k, o, d, w.hit_t[s], hit);
    const DMat& mat = sc.mats[hit.material];
    const dv3 le = (mat.kind == kEmissive && hit.front_face) ? L3(mat.color) : V(0, 0, 0);
    if (vmaxc(le) > 0) {
      const double prev_pdf = w.prev[3 * (size_t)c + s];
      const double wt =
          prev_pdf > 0 ? power_weight(prev_pdf, lights_pdf_hit(sc, ld3(w.prev, c, s, 0), hit.point)) : 1.0;
      rad = rad + vscale(vmul(tp, le), wt);
    }
    bool pending = false;
    if (mat.kind == kLambertian && p.use_nee) { /* directLight, render.zig:46-56 */
      dv3 ldir, lrad;
      double ldist, lpdf;
      if (lights_sample(sc, hit.point, rng, ldir, ldist, lrad, lpdf)) {
        const double cos_s = vdot(hit.normal, ldir);
        if (!(cos_s <= 0 || !(lpdf > 0))) {
          const double bsdf_pdf = cos_s / kPi;
          const double scale = cos_s / (kPi * lpdf) * power_weight(lpdf, bsdf_pdf);
          const dv3 direct = vscale(vmul(L3(mat.color), lrad), scale);
          double* nee = w.nee;
          st3(nee, c, s, 0, hit.point);
          st3(nee, c, s, 3, ldir);
          nee[6 * (size_t)c + s] = ldist * (1 - 1e-6);
          st3(nee, c, s, 7, direct);
          st3(nee, c, s, 10, tp);
          pending = true;
        }
      }
      if (!pending) rad = rad + vmul(tp, V(0, 0, 0)); /* directLight returned zero */
    }
    dv3 atten, sd;
    bool alive = material_scatter(mat, d, hit, rng, atten, sd);
    uint32_t depth = w.depth[s];
    if (alive) {
      tp = vmul(tp, atten);
      const double prev_pdf = (p.use_nee && mat.kind == kLambertian) ? fmax(vdot(sd, hit.normal), 0.0) / kPi : 0;
      st3(w.prev, c, s, 0, hit.point);
      w.prev[3 * (size_t)c + s] = prev_pdf;
      st3(w.ray, c, s, 0, hit.point);
      st3(w.ray, c, s, 3, sd);
      if (depth + 1 >= kRouletteDepth) { /* render.zig:94-99 */
        const double pr = fmin(vmaxc(tp), 0.95);
        if (pr <= 0 || rng_float(rng) >= pr) alive = false;
        else tp = vdiv(tp, pr);
      }
      depth += 1;
      if (alive && (uint64_t)depth >= p.max_depth) alive = false; /* loop condition, render.zig:72 */
      st3(w.tp, c, s, 0, tp);
      w.depth[s] = depth;
    }
    st3(w.rad, c, s, 0, rad);
    st_rng(w, s, rng);
    if (pending) {
      w.flags[s] = alive ? 0u : 1u;
      push(w.shadow_q, &w.ctl[kCtlShadow], s);
      if (alive) push(qn, nn, s);
    } else if (alive) {
      push(qn, nn, s);
    } else {
      finish_sample(w, p, s, rng, out, qn, nn);
    }
  }
}

/* Visibility of the light samples (render.zig:50-51) and the deferred NEE
 * add; finishes paths that ended with a sample pending. */
__global__ void __launch_bounds__(128) k_wf_shadow(DevScene sc, RenderParams p, WfState w, double* __restrict__ out) {
  const uint32_t nxt = (w.ctl[kCtlIter] & 1) ^ 1;
  const uint32_t n = w.ctl[kCtlShadow];
  uint32_t* qn = w.queue[nxt];
  uint32_t* nn = &w.ctl[kCtlExt0 + nxt];
  const uint32_t c = w.capacity;
  const double* __restrict__ nee = w.nee;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = w.shadow_q[i];
    const bool occluded = scene_occluded(sc, ld3(nee, c, s, 0), ld3(nee, c, s, 3), kRayEpsilon, nee[6 * (size_t)c + s]);
    const dv3 direct = occluded ? V(0, 0, 0) : ld3(nee, c, s, 7);
    const dv3 rad = ld3(w.rad, c, s, 0) + vmul(ld3(nee, c, s, 10), direct);
    st3(w.rad, c, s, 0, rad);
    if (w.flags[s] & 1u) {
      Rng rng = ld_rng(w, s);
      finish_sample(w, p, s, rng, out, qn, nn);
    }
  }
}

/* Queue sort, step 1: the bucket of every entry of the next extension queue
 * (direction octant, Morton cell of the origin) and per-bucket counts (a
 * shared-memory histogram per block, added to the global counts). */
__global__ void __launch_bounds__(256) k_wf_sort_keys(DevScene sc, WfState w) {
  __shared__ uint32_t hist[kSortBuckets];
  for (uint32_t i = threadIdx.x; i < kSortBuckets; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const uint32_t nxt = (w.ctl[kCtlIter] & 1) ^ 1;
  const uint32_t n = w.ctl[kCtlExt0 + nxt];
  const uint32_t* __restrict__ q = w.queue[nxt];
  const uint32_t c = w.capacity;
  const double cells = (double)(1u << kSortCellBits);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t s = q[i];
    const dv3 o = ld3(w.ray, c, s, 0), d = ld3(w.ray, c, s, 3);
    const uint32_t oct = (d.x < 0 ? 1u : 0u) | (d.y < 0 ? 2u : 0u) | (d.z < 0 ? 4u : 0u);
    uint32_t cell[3];
    const double oo[3] = {o.x, o.y, o.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double ext = sc.root_hi[a] - sc.root_lo[a];
      const double f = ext > 0 ? (oo[a] - sc.root_lo[a]) / ext * cells : 0.0;
      cell[a] = f >= cells ? (1u << kSortCellBits) - 1 : (f > 0 ? (uint32_t)f : 0u); /* NaN -> 0 */
    }
    uint32_t morton = 0;
#pragma unroll
    for (uint32_t b = 0; b < kSortCellBits; ++b)
      morton |= (((cell[0] >> b) & 1u) << (3 * b)) | (((cell[1] >> b) & 1u) << (3 * b + 1)) |
                (((cell[2] >> b) & 1u) << (3 * b + 2));
    const uint32_t key = (oct << (3 * kSortCellBits)) | morton;
    w.sort_key[i] = key;
    atomicAdd(&hist[key], 1u);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < kSortBuckets; i += blockDim.x)
    if (hist[i]) atomicAdd(&w.sort_hist[i], hist[i]);
}

/* Step 2: counts -> exclusive offsets (one block of 1024 threads, 4 buckets
 * per thread). */
__global__ void __launch_bounds__(1024) k_wf_sort_scan(WfState w) {
  __shared__ uint32_t part[1024];
  constexpr uint32_t per = kSortBuckets / 1024;
  uint32_t v[per], sum = 0;
#pragma unroll
  for (uint32_t k = 0; k < per; ++k) {
    v[k] = w.sort_hist[threadIdx.x * per + k];
    sum += v[k];
  }
  part[threadIdx.x] = sum;
  __syncthreads();
  for (uint32_t off = 1; off < 1024; off <<= 1) { /* inclusive scan of the per-thread sums */
    const uint32_t add = threadIdx.x >= off ? part[threadIdx.x - off] : 0u;
    __syncthreads();
    part[threadIdx.x] += add;
    __syncthreads();
  }
  uint32_t run = part[threadIdx.x] - sum;
#pragma unroll
  for (uint32_t k = 0; k < per; ++k) {
    w.sort_hist[threadIdx.x * per + k] = run;
    run += v[k];
  }
}

/* Step 3: every entry to its place (warp-aggregated per bucket); the order
 * within a bucket is arbitrary, which changes nothing: paths are
 * independent and each pixel belongs to one slot at a time. */
__global__ void __launch_bounds__(256) k_wf_sort_scatter(WfState w) {
  const uint32_t nxt = (w.ctl[kCtlIter] & 1) ^ 1;
  const uint32_t n = w.ctl[kCtlExt0 + nxt];
  const uint32_t* __restrict__ q = w.queue[nxt];
  const uint32_t lane = threadIdx.x & 31;
  for (uint32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    const bool live = i < n;
    const uint32_t key = live ? w.sort_key[i] : 0xFFFFFFFFu;
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    if (live) {
      const int leader = __ffs(peers) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(&w.sort_hist[key], (uint32_t)__popc(peers));
      base = __shfl_sync(peers, base, leader);
      w.sort_tmp[base + __popc(peers & ((1u << lane) - 1))] = q[i];
    }
  }
}

/* Step 4: the sorted queue back in place; counts cleared for the next sort. */
__global__ void __launch_bounds__(256) k_wf_sort_copy(WfState w) {
  const uint32_t nxt = (w.ctl[kCtlIter] & 1) ^ 1;
  const uint32_t n = w.ctl[kCtlExt0 + nxt];
  uint32_t* q = w.queue[nxt];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) q[i] = w.sort_tmp[i];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kSortBuckets; i += gridDim.x * blockDim.x)
    w.sort_hist[i] = 0;
}

/* k_wf_advance for the host-driven loop: the condition goes to ctl[kCtlGo]. */
__global__ void k_wf_advance_host(WfState w, uint64_t max_iter) {
  const uint32_t it = w.ctl[kCtlIter];
  const uint32_t nxt = (it & 1) ^ 1;
  const uint32_t n_next = w.ctl[kCtlExt0 + nxt];
  w.ctl[kCtlExt0 + (it & 1)] = 0;
  w.ctl[kCtlShadow] = 0;
  w.ctl[kCtlIter] = it + 1;
  bool go = n_next > 0;
  if (go && (uint64_t)it + 1 >= max_iter) {
    w.ctl[kCtlError] = 1;
    go = false;
  }
  w.ctl[kCtlGo] = go ? 1u : 0u;
}

/* Swaps the queues and sets the while-node condition.  The loop provably
 * ends (every active slot advances one bounce per iteration); max_iter is a
 * guard that reports an error instead of looping. */
__global__ void k_wf_advance(WfState w, cudaGraphConditionalHandle h, uint64_t max_iter) {
  const uint32_t it = w.ctl[kCtlIter];
  const uint32_t nxt = (it & 1) ^ 1;
  const uint32_t n_next = w.ctl[kCtlExt0 + nxt];
  w.ctl[kCtlExt0 + (it & 1)] = 0;
  w.ctl[kCtlShadow] = 0;
  w.ctl[kCtlIter] = it + 1;
  bool go = n_next > 0;
  if (go && (uint64_t)it + 1 >= max_iter) {
    w.ctl[kCtlError] = 1;
    go = false;
  }
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

/* meanRadiance's loop (render.zig:290-302): one thread, one RNG stream, n
 * paths along the same ray in sequence. */
__global__ void k_trace_paths(DevScene sc, double ox, double oy, double oz, double dx, double dy, double dz,
                              uint64_t* __restrict__ rng_state, uint64_t n, uint64_t max_depth, uint32_t use_nee,
                              double* __restrict__ out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  Rng rng{rng_state[0], rng_state[1], rng_state[2], rng_state[3]};
  for (uint64_t i = 0; i < n; ++i) {
    const dv3 c = trace_with<false>(sc, V(ox, oy, oz), V(dx, dy, dz), rng, max_depth, use_nee != 0, nullptr);
    out[3 * i + 0] = c.x;
    out[3 * i + 1] = c.y;
    out[3 * i + 2] = c.z;
  }
  rng_state[0] = rng.s0;
  rng_state[1] = rng.s1;
  rng_state[2] = rng.s2;
  rng_state[3] = rng.s3;
}

static int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
    if (cached <= 0) cached = 1;
  }
  return cached;
}

template <typename K>
static unsigned persistent_grid(K kernel, int block, uint64_t work_items, size_t smem = 0) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  uint64_t blocks = (uint64_t)sm_count() * per_sm;
  const uint64_t need = (work_items + block - 1) / block;
  if (blocks > need) blocks = need;
  return (unsigned)(blocks > 0 ? blocks : 1);
}

/* Megakernel variants: the nested kernel and path regeneration.  AUTO takes
 * regeneration when the upload-time pilot's mean path length reaches
 * kRegenMeanPath. */
enum MegaVariant { kMegaNested = 0, kMegaRegen = 1 };
constexpr double kRegenMeanPath = 3.0;

template <int BS, bool kFast>
static void launch_mega_bsf(const DevScene& v, const RenderParams& p, double* d_out, unsigned int* counter,
                            MegaVariant variant, cudaStream_t stream) {
  const uint64_t npix = p.width * p.rows;
  if (variant == kMegaRegen)
    k_render_regen<BS, kFast><<<persistent_grid(k_render_regen<BS, kFast>, BS, npix), BS, 0, stream>>>(v, p, d_out,
                                                                                                      counter);
  else if (p.use_nee)
    k_render_mega<BS, true, kFast><<<persistent_grid(k_render_mega<BS, true, kFast>, BS, npix), BS, 0, stream>>>(
        v, p, d_out, counter);
  else
    k_render_mega<BS, false, kFast><<<persistent_grid(k_render_mega<BS, false, kFast>, BS, npix), BS, 0, stream>>>(
        v, p, d_out, counter);
}

template <int BS>
static void launch_mega_bs(const DevScene& v, const RenderParams& p, double* d_out, unsigned int* counter,
                           MegaVariant variant, bool fast, cudaStream_t stream) {
  if (fast) launch_mega_bsf<BS, true>(v, p, d_out, counter, variant, stream);
  else launch_mega_bsf<BS, false>(v, p, d_out, counter, variant, stream);
}

static bool valid_block_size(uint32_t bs) { return bs == 0 || bs == 64 || bs == 128 || bs == 256; }

/* Whether a render takes the fast traversal: asked for, the scene has its
 * float records (a scene whose leaves or bounds do not fit them renders
 * with the f64 traversal) and, for a single render, at least
 * kFastMinPrimitives bounded primitives.  The camera origin must be within
 * the records' coordinate range as well. */
constexpr uint32_t kFastMinPrimitives = 64;
static bool use_fast(const zt_scene* s, const RenderParams& p, uint32_t precision, bool small_scenes_exact = true) {
  if (precision != ZT_PRECISION_FAST || !s->device || !s->device->view.fast_ok) return false;
  /* on a tree this small the float walk's per-ray set-up costs more than its
   * box tests save (Cornell box, 14 primitives: 477 vs 565 Msamples/s); a
   * batch, whose renders share one kernel instance, skips this rule */
  if (small_scenes_exact && s->device->view.n_prims < kFastMinPrimitives) return false;
  const double* o = p.cam.origin;
  const double reach = fabs(p.cam.lens_radius) * (fabs(p.cam.u[0]) + fabs(p.cam.u[1]) + fabs(p.cam.u[2]) +
                                                  fabs(p.cam.v[0]) + fabs(p.cam.v[1]) + fabs(p.cam.v[2]));
  return fabs(o[0]) + reach <= kFastMaxCoord && fabs(o[1]) + reach <= kFastMaxCoord &&
         fabs(o[2]) + reach <= kFastMaxCoord;
}

static zt_status launch_mega(zt_scene* s, const RenderParams& p, uint32_t block_size, double* d_out,
                             MegaVariant variant, bool fast, cudaStream_t stream) {
  zt_device_buffers* d = s->device;
  ZT_CUDA(cudaMemsetAsync(d->counter, 0, sizeof(unsigned int), stream), "reset work counter");
  const DevScene v = launch_view(s);
  if (block_size == 64) launch_mega_bs<64>(v, p, d_out, d->counter, variant, fast, stream);
  else if (block_size == 256) launch_mega_bs<256>(v, p, d_out, d->counter, variant, fast, stream);
  else launch_mega_bs<128>(v, p, d_out, d->counter, variant, fast, stream);
  ZT_CUDA(cudaGetLastError(), "launch the megakernel");
  return ZT_OK;
}

/* Carves the wavefront arrays out of one allocation of `cap` slots. */
static zt_status wavefront_state(zt_device_buffers* d, uint32_t cap) {
  zt_wavefront_cache& c = d->wf;
  if (c.block && c.capacity >= cap) return ZT_OK;
  if (c.done) cudaEventSynchronize(c.done);
  if (c.exec) { cudaGraphExecDestroy(c.exec); c.exec = nullptr; }
  cudaFree(c.block);
  c.block = nullptr;
  c.capacity = 0;
  const size_t n = cap;
  const size_t sizes[] = {4 * n, 4 * n, 4 * n, 4 * n, 32 * n, 48 * n, 24 * n, 24 * n, 24 * n, 32 * n,
                          8 * n, 4 * n, 104 * n, 4 * n, 4 * n, 4 * n, 64, 4 * n, 4 * n, 4 * kSortBuckets};
  size_t offs[20], cur = 0;
  for (int i = 0; i < 20; ++i) { offs[i] = cur; cur = align256(cur + sizes[i]); }
  ZT_CUDA(cudaMalloc(&c.block, cur), "allocate wavefront state");
  char* b = (char*)c.block;
  WfState& w = c.state;
  w.pix = (uint32_t*)(b + offs[0]);
  w.sample = (uint32_t*)(b + offs[1]);
  w.depth = (uint32_t*)(b + offs[2]);
  w.flags = (uint32_t*)(b + offs[3]);
  w.rng = (uint64_t*)(b + offs[4]);
  w.ray = (double*)(b + offs[5]);
  w.tp = (double*)(b + offs[6]);
  w.rad = (double*)(b + offs[7]);
  w.sum = (double*)(b + offs[8]);
  w.prev = (double*)(b + offs[9]);
  w.hit_t = (double*)(b + offs[10]);
  w.hit_k = (int32_t*)(b + offs[11]);
  w.nee = (double*)(b + offs[12]);
  w.queue[0] = (uint32_t*)(b + offs[13]);
  w.queue[1] = (uint32_t*)(b + offs[14]);
  w.shadow_q = (uint32_t*)(b + offs[15]);
  w.ctl = (uint32_t*)(b + offs[16]);
  w.sort_key = (uint32_t*)(b + offs[17]);
  w.sort_tmp = (uint32_t*)(b + offs[18]);
  w.sort_hist = (uint32_t*)(b + offs[19]);
  ZT_CUDA(cudaMemset(w.sort_hist, 0, 4 * kSortBuckets), "clear the queue sort's counts");
  w.capacity = cap;
  c.bytes = cur;
  c.capacity = cap;
  return ZT_OK;
}

/* Builds the executable graph: while (queue not empty) { extend; shade;
 * shadow; advance }.  The loop runs on the device; the host never waits. */
/* One iteration's kernels after the intersection: shade, shadow and, for
 * the sorted form, the four queue-sort kernels. */
static void enqueue_wavefront_step(const DevScene& view, const RenderParams& p, const WfState& w, double* d_out,
                                   bool sorted, cudaStream_t cs) {
  const uint64_t cap = w.capacity;
  k_wf_extend<<<persistent_grid(k_wf_extend, 128, cap), 128, 0, cs>>>(view, w);
  k_wf_shade<<<persistent_grid(k_wf_shade, 128, cap), 128, 0, cs>>>(view, p, w, d_out);
  k_wf_shadow<<<persistent_grid(k_wf_shadow, 128, cap), 128, 0, cs>>>(view, p, w, d_out);
  if (sorted) {
    k_wf_sort_keys<<<persistent_grid(k_wf_sort_keys, 256, cap), 256, 0, cs>>>(view, w);
    k_wf_sort_scan<<<1, 1024, 0, cs>>>(w);
    k_wf_sort_scatter<<<persistent_grid(k_wf_sort_scatter, 256, cap), 256, 0, cs>>>(w);
    k_wf_sort_copy<<<persistent_grid(k_wf_sort_copy, 256, cap), 256, 0, cs>>>(w);
  }
}

static zt_status build_wavefront_graph(const DevScene& view, const RenderParams& p, const WfState& w, double* d_out,
                                       uint64_t max_iter, bool sorted, cudaGraphExec_t* exec_out) {
  cudaGraph_t g = nullptr;
  cudaStream_t cs = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  cudaGraphConditionalHandle h;
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) {
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      enqueue_wavefront_step(view, p, w, d_out, sorted, cs);
      k_wf_advance<<<1, 1, 0, cs>>>(w, h, max_iter);
      cudaGraph_t captured = nullptr;
      cudaError_t e2 = cudaStreamEndCapture(cs, &captured);
      e = e2 != cudaSuccess ? e2 : cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
  if (cs) cudaStreamDestroy(cs);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) return cuda_fail(e, "build wavefront graph");
  *exec_out = exec;
  return ZT_OK;
}

/* Iteration bound of the wavefront loop: every iteration advances each
 * active slot by one bounce, so pixels x spp x (max_depth + 1) iterations
 * finish any render; g_wf_iteration_limit (zt_set_wavefront_iteration_limit)
 * can lower it to exercise the bound's error path. */
static std::atomic<uint64_t> g_wf_iteration_limit{0};

static uint64_t wavefront_max_iter(const RenderParams& p) {
  const double bound = (double)(p.width * p.height) * (double)p.spp * (double)(p.max_depth + 1) + 16.0;
  uint64_t max_iter = bound > 4.0e9 ? 4000000000ull : (uint64_t)bound;
  const uint64_t lim = g_wf_iteration_limit.load();
  if (lim && lim < max_iter) max_iter = lim;
  return max_iter;
}

/* The same loop driven from the host, one synchronisation per iteration,
 * when ZT_WAVEFRONT_HOST_LOOP is set in the environment: profilers that do
 * not see kernels inside a conditional graph node can then measure the
 * wavefront kernels one launch at a time.  Same kernels, same pixels. */
static zt_status run_wavefront_host_loop(const DevScene& view, const RenderParams& p, const WfState& w,
                                         double* d_out, uint64_t max_iter, bool sorted, cudaStream_t stream) {
  for (;;) {
    enqueue_wavefront_step(view, p, w, d_out, sorted, stream);
    k_wf_advance_host<<<1, 1, 0, stream>>>(w, max_iter);
    uint32_t go = 0;
    ZT_CUDA(cudaMemcpyAsync(&go, w.ctl + kCtlGo, sizeof go, cudaMemcpyDeviceToHost, stream), "read loop condition");
    ZT_CUDA(cudaStreamSynchronize(stream), "wavefront iteration");
    if (!go) return ZT_OK;
  }
}

static zt_status launch_wavefront(zt_scene* s, const RenderParams& p, uint32_t capacity, bool sorted, double* d_out,
                                  cudaStream_t stream) {
  zt_device_buffers* d = s->device;
  const uint64_t npix = p.width * p.height;
  const uint32_t cap = (uint32_t)(capacity && capacity < npix ? capacity : (npix < (1u << 22) ? npix : (1u << 22)));
  zt_status rc = wavefront_state(d, cap);
  if (rc != ZT_OK) return rc;
  zt_wavefront_cache& c = d->wf;
  const DevScene view = launch_view(s);
  unsigned char key[sizeof c.key];
  memset(key, 0, sizeof key);
  memcpy(key, &view, sizeof view);
  memcpy(key + sizeof view, &p, sizeof p);
  memcpy(key + sizeof view + sizeof p, &d_out, sizeof d_out);
  const uint64_t capk = cap | (sorted ? 1ull << 40 : 0ull), max_iter = wavefront_max_iter(p);
  memcpy(key + sizeof view + sizeof p + sizeof d_out, &capk, sizeof capk);
  memcpy(key + sizeof view + sizeof p + sizeof d_out + sizeof capk, &max_iter, sizeof max_iter);
  const uint32_t n0 = (uint32_t)(npix < cap ? npix : cap);
  if (getenv("ZT_WAVEFRONT_HOST_LOOP")) {
    k_wf_init<<<persistent_grid(k_wf_init, 256, n0), 256, 0, stream>>>(p, c.state, n0);
    ZT_CUDA(cudaGetLastError(), "launch k_wf_init");
    return run_wavefront_host_loop(view, p, c.state, d_out, max_iter, sorted, stream);
  }
  if (!c.exec || memcmp(key, c.key, sizeof key) != 0) {
    if (c.done) cudaEventSynchronize(c.done);
    if (c.exec) { cudaGraphExecDestroy(c.exec); c.exec = nullptr; }
    rc = build_wavefront_graph(view, p, c.state, d_out, max_iter, sorted, &c.exec);
    if (rc != ZT_OK) return rc;
    memcpy(c.key, key, sizeof key);
    if (!c.done) ZT_CUDA(cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming), "create event");
  }
  k_wf_init<<<persistent_grid(k_wf_init, 256, n0), 256, 0, stream>>>(p, c.state, n0);
  ZT_CUDA(cudaGetLastError(), "launch k_wf_init");
  ZT_CUDA(cudaGraphLaunch(c.exec, stream), "launch wavefront graph");
  ZT_CUDA(cudaEventRecord(c.done, stream), "record event");
  return ZT_OK;
}

/* Renders the rows [p.row0, p.row0 + p.rows) of the image into d_out (the
 * band's rows only).  The wavefront mode renders whole images. */
static zt_status launch_render_params(zt_scene* s, const RenderParams& p, const zt_gpu_config* cfg, double* d_out,
                                      cudaStream_t stream) {
  if (p.max_depth == 0) { /* traceWith never enters its loop: every sample is zero */
    ZT_CUDA(cudaMemsetAsync(d_out, 0, p.width * p.rows * 3 * sizeof(double), stream), "clear framebuffer");
    return ZT_OK;
  }
  const uint32_t mode = cfg ? cfg->mode : ZT_MODE_AUTO;
  if (mode == ZT_MODE_WAVEFRONT || mode == ZT_MODE_WAVEFRONT_SORTED) {
    if (p.row0 != 0 || p.rows != p.height)
      return fail(ZT_ERR_INVALID_ARGUMENT, "the wavefront mode renders whole images, not row bands");
    return launch_wavefront(s, p, cfg ? cfg->queue_capacity : 0, mode == ZT_MODE_WAVEFRONT_SORTED, d_out, stream);
  }
  if (mode > ZT_MODE_MEGAKERNEL_REGEN) return fail(ZT_ERR_INVALID_ARGUMENT, "unknown zt_gpu_config.mode");
  const uint32_t bs = cfg ? cfg->block_size : 0;
  if (!valid_block_size(bs)) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_gpu_config.block_size must be 0, 64, 128 or 256");
  const uint32_t precision = cfg ? cfg->precision : ZT_PRECISION_EXACT;
  if (precision > ZT_PRECISION_FAST) return fail(ZT_ERR_INVALID_ARGUMENT, "unknown zt_gpu_config.precision");
  const bool long_paths = s->pilot_valid && s->mean_path >= kRegenMeanPath;
  const MegaVariant variant =
      (mode == ZT_MODE_MEGAKERNEL_REGEN || (mode == ZT_MODE_AUTO && long_paths)) ? kMegaRegen : kMegaNested;
  return launch_mega(s, p, bs, d_out, variant, use_fast(s, p, precision), stream);
}

static zt_status launch_render(zt_scene* s, const zt_options* o, const zt_gpu_config* cfg, double* d_out,
                               cudaStream_t stream) {
  return launch_render_params(s, make_params(s, o), cfg, d_out, stream);
}

/* Error word of the last wavefront launch (after the stream is idle). */
static zt_status wavefront_status(zt_scene* s, const zt_gpu_config* cfg) {
  if (!cfg || (cfg->mode != ZT_MODE_WAVEFRONT && cfg->mode != ZT_MODE_WAVEFRONT_SORTED) || !s->device ||
      !s->device->wf.block)
    return ZT_OK;
  uint32_t err = 0;
  ZT_CUDA(cudaMemcpy(&err, s->device->wf.state.ctl + kCtlError, sizeof err, cudaMemcpyDeviceToHost), "read status");
  if (err) return fail(ZT_ERR_TIMEOUT, "wavefront loop exceeded its iteration bound");
  return ZT_OK;
}

static zt_status check_render_args(zt_scene* s, const zt_options* o) {
  if (!s || !o) return fail(ZT_ERR_INVALID_ARGUMENT, "NULL scene or options");
  if (!options_valid(o)) return fail(ZT_ERR_INVALID_OPTIONS, "InvalidOptions: width, height, spp and tile_size must be > 0");
  if (o->width > (1ull << 31) || o->height > (1ull << 31) || o->width * o->height > (1ull << 31))
    return fail(ZT_ERR_INVALID_OPTIONS, "InvalidOptions: more than 2^31 pixels");
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built: call zt_scene_build first");
  return ZT_OK;
}

}  // namespace zt

extern "C" {

zt_status zt_scene_upload(zt_scene* s) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_upload: NULL scene");
  return upload(s);
}

zt_status zt_scene_upload_bytes(zt_scene* s, uint64_t* bytes) {
  if (!s || !bytes) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_upload_bytes: NULL argument");
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built: call zt_scene_build first");
  zt_status rc = make_staging(s);
  if (rc != ZT_OK) return rc;
  *bytes = s->staging->bytes;
  return ZT_OK;
}

zt_status zt_scene_release_device(zt_scene* s) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_release_device: NULL scene");
  release_device(s);
  return ZT_OK;
}

zt_status zt_render_device(zt_scene* s, const zt_options* o, const zt_gpu_config* cfg, double* d_out, void* stream) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!d_out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_device: NULL output");
  int dev = 0;
  ZT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (!s->device || s->device->device != dev)
    return fail(ZT_ERR_INVALID_ARGUMENT, "scene is not resident on the current device: call zt_scene_upload");
  return launch_render(s, o, cfg, d_out, (cudaStream_t)stream);
}

zt_status zt_set_wavefront_iteration_limit(uint64_t max_iterations) {
  g_wf_iteration_limit.store(max_iterations);
  return ZT_OK;
}

zt_status zt_render_rows_device(zt_scene* s, const zt_options* o, uint64_t row_begin, uint64_t row_end,
                                const zt_gpu_config* cfg, double* d_out, void* stream) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!d_out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_rows_device: NULL output");
  if (row_begin >= row_end || row_end > o->height)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_rows_device: need row_begin < row_end <= height");
  int dev = 0;
  ZT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (!s->device || s->device->device != dev)
    return fail(ZT_ERR_INVALID_ARGUMENT, "scene is not resident on the current device: call zt_scene_upload");
  RenderParams p = make_params(s, o); /* camera and RNG streams of the whole image */
  p.row0 = row_begin;
  p.rows = row_end - row_begin;
  return launch_render_params(s, p, cfg, d_out, (cudaStream_t)stream);
}

zt_status zt_render_ex(zt_scene* s, const zt_options* o, const zt_gpu_config* cfg, double* out) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render: NULL output");
  rc = upload(s);
  if (rc != ZT_OK) return rc;
  const size_t bytes = (size_t)(o->width * o->height * 3) * sizeof(double);
  double* d_out = nullptr;
  if ((rc = pool_alloc((void**)&d_out, bytes, 0, "allocate framebuffer")) != ZT_OK) return rc;
  rc = launch_render(s, o, cfg, d_out, 0);
  if (rc == ZT_OK) {
    cudaError_t e = cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) rc = cuda_fail(e, "render / copy framebuffer");
    else rc = wavefront_status(s, cfg);
  }
  pool_free(d_out, 0);
  return rc;
}

zt_status zt_render(zt_scene* s, const zt_options* o, double* out) { return zt_render_ex(s, o, nullptr, out); }

/* Render, encode and (for PNG) assemble the file on the device; only the
 * encoded bytes cross PCIe.  One device allocation holds the framebuffer,
 * the RGB8 image, the PNG and its checksum scratch. */
static zt_status render_encoded(zt_scene* s, const zt_options* o, const zt_gpu_config* cfg, uint32_t tonemap,
                                double gamma, double exposure, bool png, uint8_t* out, uint64_t capacity) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!out) return fail(ZT_ERR_INVALID_ARGUMENT, "NULL output");
  if (tonemap > 2) return fail(ZT_ERR_INVALID_ARGUMENT, "tonemap must be 0 (none), 1 (reinhard) or 2 (aces)");
  PngLayout L{};
  const uint64_t npix = o->width * o->height;
  uint64_t out_bytes = 3 * npix;
  if (png) {
    if ((rc = zt_png_size(o->width, o->height, &out_bytes)) != ZT_OK) return rc;
    L = png_layout(o->width, o->height);
  }
  if (capacity < out_bytes) return fail(ZT_ERR_INVALID_ARGUMENT, "output buffer too small");
  if ((rc = upload(s)) != ZT_OK) return rc;
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t fb_bytes = up(npix * 3 * sizeof(double)), rgb_bytes = up(npix * 3);
  const size_t png_bytes = png ? up(L.total) : 0, scratch_bytes = png ? up(png_scratch_bytes(L)) : 0;
  unsigned char* block = nullptr;
  if ((rc = pool_alloc((void**)&block, fb_bytes + rgb_bytes + png_bytes + scratch_bytes, 0,
                       "allocate output buffers")) != ZT_OK)
    return rc;
  double* d_fb = reinterpret_cast<double*>(block);
  uint8_t* d_rgb = block + fb_bytes;
  uint8_t* d_png = d_rgb + rgb_bytes;
  rc = launch_render(s, o, cfg, d_fb, 0);
  if (rc == ZT_OK) rc = launch_encode_rgb8(d_fb, 3 * npix, tonemap, gamma, exposure, d_rgb, 0);
  if (rc == ZT_OK && png) rc = launch_png(d_rgb, L, d_png, d_png + png_bytes, 0);
  if (rc == ZT_OK) {
    cudaError_t e = cudaMemcpyAsync(out, png ? d_png : d_rgb, out_bytes, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) rc = cuda_fail(e, "copy encoded image");
    else rc = wavefront_status(s, cfg);
  }
  pool_free(block, 0);
  return rc;
}

zt_status zt_render_rgb8(zt_scene* s, const zt_options* o, const zt_gpu_config* cfg, uint32_t tonemap, double gamma,
                         double exposure, uint8_t* rgb_out) {
  if (!o) return fail(ZT_ERR_INVALID_ARGUMENT, "NULL options");
  return render_encoded(s, o, cfg, tonemap, gamma, exposure, false, rgb_out, o->width * o->height * 3);
}

zt_status zt_render_png(zt_scene* s, const zt_options* o, const zt_gpu_config* cfg, uint32_t tonemap, double gamma,
                        double exposure, uint8_t* png_out, uint64_t png_capacity) {
  return render_encoded(s, o, cfg, tonemap, gamma, exposure, true, png_out, png_capacity);
}

zt_status zt_render_rows(zt_scene* s, const zt_options* o, uint64_t row_begin, uint64_t row_end, double* out) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_rows: NULL output");
  if (row_begin >= row_end || row_end > o->height)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_rows: need row_begin < row_end <= height");
  if ((rc = upload(s)) != ZT_OK) return rc;
  RenderParams p = make_params(s, o); /* camera and RNG streams of the whole image */
  p.row0 = row_begin;
  p.rows = row_end - row_begin;
  const size_t bytes = (size_t)(p.rows * p.width * 3) * sizeof(double);
  if (p.max_depth == 0) {
    memset(out, 0, bytes);
    return ZT_OK;
  }
  double* d_out = nullptr;
  if ((rc = pool_alloc((void**)&d_out, bytes, 0, "allocate framebuffer band")) != ZT_OK) return rc;
  rc = launch_mega(s, p, 0, d_out, s->pilot_valid && s->mean_path >= kRegenMeanPath ? kMegaRegen : kMegaNested,
                   false, 0);
  if (rc == ZT_OK) {
    cudaError_t e = cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) rc = cuda_fail(e, "render rows / copy framebuffer band");
  }
  pool_free(d_out, 0);
  return rc;
}

/* Pilot for ZT_MODE_AUTO, run by the synchronous entry points (upload)
 * once per build, camera and background: the mean path length of one sample
 * per pixel of a 64x64 image from the scene's camera (depth 16).  Long paths
 * (closed scenes) favour the path-regeneration megakernel: on the Cornell box
 * (mean 3.4) it is 1.5x the nested one, on open scenes (random spheres 2.5,
 * the 1M-triangle terrain 1.6) 0.95x and 0.86x. */
}  /* extern "C" */

namespace zt {
static zt_status pilot_paths(zt_scene* s) {
  zt_options o;
  memset(&o, 0, sizeof o);
  o.width = o.height = 64;
  o.spp = 1;
  o.max_depth = 16;
  o.threads = 1;
  o.tile_size = 16;
  o.light_sampling = 1;
  const uint64_t npix = o.width * o.height;
  int32_t* d_fp = nullptr;
  uint32_t* d_pl = nullptr;
  ZT_CUDA(cudaMalloc((void**)&d_fp, npix * (sizeof(int32_t) + sizeof(uint32_t))), "allocate pilot buffer");
  d_pl = reinterpret_cast<uint32_t*>(d_fp + npix);
  const RenderParams p = make_params(s, &o);
  k_render_debug<<<(unsigned)((npix + 127) / 128), 128>>>(launch_view(s), p, d_fp, d_pl);
  std::vector<uint32_t> pl(npix);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(pl.data(), d_pl, npix * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(d_fp);
  if (e != cudaSuccess) return cuda_fail(e, "pilot render");
  double sum = 0;
  for (uint32_t v : pl) sum += v;
  s->mean_path = sum / (double)npix;
  s->pilot_valid = true;
  return ZT_OK;
}
}  // namespace zt

extern "C" {

zt_status zt_render_debug(zt_scene* s, const zt_options* o, int32_t* first_prim, uint32_t* path_len) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!first_prim || !path_len) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_debug: NULL output");
  rc = upload(s);
  if (rc != ZT_OK) return rc;
  const uint64_t npix = o->width * o->height;
  int32_t* d_fp = nullptr;
  uint32_t* d_pl = nullptr;
  ZT_CUDA(cudaMalloc((void**)&d_fp, npix * sizeof(int32_t)), "allocate debug buffer");
  cudaError_t e = cudaMalloc((void**)&d_pl, npix * sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaFree(d_fp);
    return cuda_fail(e, "allocate debug buffer");
  }
  const RenderParams p = make_params(s, o);
  k_render_debug<<<(unsigned)((npix + 127) / 128), 128>>>(launch_view(s), p, d_fp, d_pl);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(first_prim, d_fp, npix * sizeof(int32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(path_len, d_pl, npix * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  cudaFree(d_fp);
  cudaFree(d_pl);
  if (e != cudaSuccess) return cuda_fail(e, "debug render");
  return ZT_OK;
}

zt_status zt_trace_paths(zt_scene* s, const zt_vec3* origin, const zt_vec3* dir, uint64_t* rng_state, uint64_t n,
                         uint64_t max_depth, uint32_t light_sampling, double* out) {
  if (!s || !origin || !dir || !rng_state || (!out && n))
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_trace_paths: NULL argument");
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built: call zt_scene_build first");
  zt_status rc = upload(s);
  if (rc != ZT_OK) return rc;
  if (n == 0) return ZT_OK;
  uint64_t* d_rng = nullptr;
  double* d_out = nullptr;
  ZT_CUDA(cudaMalloc((void**)&d_rng, 4 * sizeof(uint64_t)), "allocate rng state");
  cudaError_t e = cudaMalloc((void**)&d_out, n * 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(d_rng, rng_state, 4 * sizeof(uint64_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    const uint32_t use_nee = (light_sampling && !s->lights.empty()) ? 1u : 0u; /* render.zig:62 */
    k_trace_paths<<<1, 32>>>(launch_view(s), origin->x, origin->y, origin->z, dir->x, dir->y, dir->z, d_rng, n,
                             max_depth, use_nee, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, n * 3 * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(rng_state, d_rng, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost);
  cudaFree(d_rng);
  cudaFree(d_out);
  if (e != cudaSuccess) return cuda_fail(e, "trace paths");
  return ZT_OK;
}

zt_status zt_rng_streams(uint64_t seed, uint64_t stream0, uint64_t n_streams, uint64_t n_draws, uint64_t* out) {
  if (!out && n_streams * n_draws) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_rng_streams: NULL output");
  if (n_streams == 0 || n_draws == 0) return ZT_OK;
  const size_t bytes = (size_t)(n_streams * n_draws) * sizeof(uint64_t);
  uint64_t* d = nullptr;
  ZT_CUDA(cudaMalloc((void**)&d, bytes), "allocate rng buffer");
  k_rng_streams<<<(unsigned)((n_streams + 127) / 128), 128>>>(seed, stream0, n_streams, n_draws, d);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(out, d, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "rng streams");
  return ZT_OK;
}

}  /* extern "C" */

/* --------------------------------------------------- Differentiable form ---- */
namespace zt {

/* Forward of the detached estimator (zt_diff.cuh): the megakernel's tile
 * loop with trace_diff; theta == the scene's colours gives zt_render's image.
 * The differentiable kernels are built for four blocks of 128 per SM (128
 * registers): their longer code spills heavily at 72 registers, and at
 * 512x512 the fewer resident warps measured faster (forward 28 vs 31 ms,
 * backward 52 vs 57-62 ms). */
template <int BS>
__global__ void __launch_bounds__(BS, 512 / BS) k_forward_diff(DevScene sc, RenderParams p,
                                                             const double* __restrict__ theta,
                                                             double* __restrict__ out, double* __restrict__ sample_L,
                                                             unsigned int* __restrict__ counter) {
  const uint64_t tiles_x = (p.width + 7) / 8, tiles = tiles_x * ((p.rows + 3) / 4);
  const uint64_t row_end = p.row0 + p.rows;
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= tiles) return;
    const uint64_t x = (tile % tiles_x) * 8 + (lane & 7), y = p.row0 + (tile / tiles_x) * 4 + (lane >> 3);
    if (x >= p.width || y >= row_end) continue;
    const uint64_t pix = y * p.width + x;
    Rng rng = rng_for_stream(p.seed, pix);
    dv3 sum = V(0, 0, 0);
    for (uint64_t i = 0; i < p.spp; ++i) {
      const double s = ((double)x + rng_float(rng)) / (double)p.width;
      const double t = ((double)y + rng_float(rng)) / (double)p.height;
      dv3 ro, rd;
      camera_ray(p.cam, s, t, rng, ro, rd);
      const dv3 c = trace_diff(sc, theta, ro, rd, rng, p.max_depth, p.use_nee != 0, false, V(0, 0, 0), V(0, 0, 0),
                               nullptr, false);
      if (sample_L) { /* the primal radiance of every sample, kept for zt_backward */
        double* q = sample_L + 3 * (i * p.width * p.height + pix);
        q[0] = c.x;
        q[1] = c.y;
        q[2] = c.z;
      }
      if (visfinite(c)) sum = sum + c;
    }
    const dv3 px = vscale(sum, 1.0 / (double)p.spp);
    const uint64_t o = pix - p.row0 * p.width; /* output starts at the band's first row */
    out[3 * o + 0] = px.x;
    out[3 * o + 1] = px.y;
    out[3 * o + 2] = px.z;
  }
}

/* Path-replay adjoint: for every sample, the primal pass gives its radiance
 * L, then the same path is replayed from the saved RNG state accumulating
 * dL/dtheta into per-block shared memory (flushed once per block), or
 * straight into global memory when the parameter table is large.  Built for
 * five blocks of 128 per SM (up to 102 registers): 50.0 against 50.8 ms at
 * four blocks (128 registers) on the 512x512x64 Cornell-style workload; the
 * forward kernel stays at four (27.5 against 28.1 ms). */
template <int BS>
__global__ void __launch_bounds__(BS, 640 / BS) k_backward_diff(DevScene sc, RenderParams p,
                                                              const double* __restrict__ theta,
                                                              const double* __restrict__ dimg, double* grad,
                                                              uint32_t n_params, int use_smem,
                                                              const double* __restrict__ sample_L,
                                                              unsigned int* __restrict__ counter) {
  extern __shared__ double sgrad[];
  double* g = use_smem ? sgrad + (threadIdx.x >> 5) * n_params : grad; /* a slice per warp */
  if (use_smem) {
    for (uint32_t i = threadIdx.x; i < n_params * (BS / 32); i += BS) sgrad[i] = 0.0;
    __syncthreads();
  }
  const uint64_t tiles_x = (p.width + 7) / 8, tiles = tiles_x * ((p.rows + 3) / 4);
  const uint64_t row_end = p.row0 + p.rows;
  const unsigned lane = threadIdx.x & 31;
  const double inv_spp = 1.0 / (double)p.spp;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= tiles) break;
    const uint64_t x = (tile % tiles_x) * 8 + (lane & 7), y = p.row0 + (tile / tiles_x) * 4 + (lane >> 3);
    if (x >= p.width || y >= row_end) continue;
    const uint64_t pix = y * p.width + x;
    /* dL/dpixel of the band (rows row0 ..), pixel = sum * (1/spp), render.zig:144 */
    const dv3 adj = vscale(L3(dimg + 3 * (pix - p.row0 * p.width)), inv_spp);
    if (adj.x == 0 && adj.y == 0 && adj.z == 0) continue;
    Rng rng = rng_for_stream(p.seed, pix);
    for (uint64_t i = 0; i < p.spp; ++i) {
      const double s = ((double)x + rng_float(rng)) / (double)p.width;
      const double t = ((double)y + rng_float(rng)) / (double)p.height;
      dv3 ro, rd;
      camera_ray(p.cam, s, t, rng, ro, rd);
      const Rng start = rng;
      dv3 L = V(0, 0, 0);
      int first_pass = 0;
      if (sample_L) { /* the forward kept the primal radiance: replay only */
        L = L3(sample_L + 3 * (i * p.width * p.height + pix));
        first_pass = 1;
        if (!visfinite(L)) { /* dropped by the forward (render.zig:142): advance the stream only */
          Rng r = start;
          trace_diff(sc, theta, ro, rd, r, p.max_depth, p.use_nee != 0, false, L, adj, g, use_smem);
          rng = r;
          continue;
        }
      }
#pragma unroll 1
      for (int pass = first_pass; pass < 2; ++pass) { /* primal, then replay from the same stream state */
        Rng r = start;
        const dv3 v = trace_diff(sc, theta, ro, rd, r, p.max_depth, p.use_nee != 0, pass == 1, L, adj, g, use_smem);
        if (pass == 0) {
          L = v;
          if (!visfinite(L)) { /* dropped by the forward (render.zig:142): no gradient */
            rng = r;
            break;
          }
        } else {
          rng = r; /* the replay draws exactly what the primal drew */
        }
      }
    }
  }
  if (use_smem) { /* sum the warps' slices, then one global add per parameter and block */
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n_params; i += BS) {
      double acc = 0.0;
      for (int wi = 0; wi < BS / 32; ++wi) acc += sgrad[wi * n_params + i];
      if (acc != 0.0) atomicAdd(grad + i, acc);
    }
  }
}

/* theta on the host: the caller's colours, or the scene's own. */
static std::vector<double> theta_host(const zt_scene* s, const double* colors) {
  std::vector<double> th(s->materials.size() * 3, 0.0);
  for (size_t m = 0; m < s->materials.size(); ++m) {
    const zt_vec3& c = s->materials[m].color;
    th[3 * m + 0] = colors ? colors[3 * m + 0] : c.x;
    th[3 * m + 1] = colors ? colors[3 * m + 1] : c.y;
    th[3 * m + 2] = colors ? colors[3 * m + 2] : c.z;
  }
  return th;
}

/* The parameters on the device, from the stream-ordered pool (legacy
 * default stream, as every per-call buffer of the differentiable pair). */
static zt_status upload_theta(const std::vector<double>& th, double** d_theta) {
  const size_t n = th.empty() ? 3 : th.size();
  zt_status rc = pool_alloc((void**)d_theta, n * sizeof(double), 0, "allocate parameters");
  if (rc != ZT_OK) return rc;
  if (!th.empty()) {
    const cudaError_t e = cudaMemcpy(*d_theta, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      pool_free(*d_theta, 0);
      *d_theta = nullptr;
      return cuda_fail(e, "upload parameters");
    }
  }
  return ZT_OK;
}

static bool same_render(const zt_options& a, const zt_options& b) {
  return a.width == b.width && a.height == b.height && a.spp == b.spp && a.max_depth == b.max_depth &&
         a.seed == b.seed && a.light_sampling == b.light_sampling;
}

}  // namespace zt

extern "C" {

zt_status zt_forward(zt_scene* s, const zt_options* o, const double* colors, double* out) {
  if (!o) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_forward: NULL options");
  return zt_forward_rows(s, o, 0, o->height, colors, out);
}

zt_status zt_forward_rows(zt_scene* s, const zt_options* o, uint64_t row_begin, uint64_t row_end,
                          const double* colors, double* out) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_forward: NULL output");
  if (row_begin >= row_end || row_end > o->height)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_forward_rows: need row_begin < row_end <= height");
  if ((rc = upload(s)) != ZT_OK) return rc;
  RenderParams p = make_params(s, o);
  p.row0 = row_begin;
  p.rows = row_end - row_begin;
  const size_t bytes = (size_t)(p.rows * o->width * 3) * sizeof(double);
  zt_diff_cache& cache = s->device->diff;
  cache.valid = false;
  if (p.max_depth == 0) {
    memset(out, 0, bytes);
    return ZT_OK;
  }
  const std::vector<double> th = theta_host(s, colors);
  double *d_theta = nullptr, *d_out = nullptr;
  if ((rc = upload_theta(th, &d_theta)) != ZT_OK) return rc;
  /* keep every sample's primal radiance for a following zt_backward (24 bytes
   * per sample of the whole image, indexed by image pixel) when that fits the
   * scene's primal cache limit; above it, or if the memory is not available,
   * the backward recomputes the primal from the RNG stream */
  const size_t n_l = (size_t)(p.width * p.height * p.spp) * 3;
  const bool keep = (uint64_t)n_l * sizeof(double) <= s->primal_cache_limit;
  if (!keep || cache.cap < n_l) {
    cudaFree(cache.L);
    cache.L = nullptr;
    cache.cap = 0;
    if (keep) {
      if (cudaMalloc((void**)&cache.L, n_l * sizeof(double)) == cudaSuccess) cache.cap = n_l;
      else cudaGetLastError();
    }
  }
  if ((rc = pool_alloc((void**)&d_out, bytes, 0, "allocate framebuffer")) != ZT_OK) {
    pool_free(d_theta, 0);
    return rc;
  }
  cudaError_t e = cudaMemsetAsync(s->device->counter, 0, sizeof(unsigned int), 0);
  if (e == cudaSuccess) {
    k_forward_diff<128><<<persistent_grid(k_forward_diff<128>, 128, p.width * p.rows), 128>>>(
        launch_view(s), p, d_theta, d_out, cache.L, s->device->counter);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost);
  pool_free(d_theta, 0);
  pool_free(d_out, 0);
  if (e != cudaSuccess) return cuda_fail(e, "zt_forward");
  if (cache.L) {
    cache.valid = true;
    cache.opts = *o;
    cache.row0 = p.row0;
    cache.rows = p.rows;
    cache.theta = th;
    cache.camera = s->camera;
    cache.background = s->background;
  }
  return ZT_OK;
}

zt_status zt_scene_set_primal_cache_limit(zt_scene* s, uint64_t max_bytes) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_set_primal_cache_limit: NULL scene");
  s->primal_cache_limit = max_bytes;
  if (s->device && s->device->diff.cap * sizeof(double) > max_bytes) { /* drop a cache above the new limit */
    zt_diff_cache& c = s->device->diff;
    cudaDeviceSynchronize();
    cudaFree(c.L);
    c.L = nullptr;
    c.cap = 0;
    c.valid = false;
  }
  return ZT_OK;
}

zt_status zt_backward(zt_scene* s, const zt_options* o, const double* colors, const double* d_image,
                      double* d_colors) {
  if (!o) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_backward: NULL options");
  return zt_backward_rows(s, o, 0, o->height, colors, d_image, d_colors);
}

zt_status zt_backward_rows(zt_scene* s, const zt_options* o, uint64_t row_begin, uint64_t row_end,
                           const double* colors, const double* d_image, double* d_colors) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!d_image || !d_colors) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_backward: NULL argument");
  if (row_begin >= row_end || row_end > o->height)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_backward_rows: need row_begin < row_end <= height");
  if ((rc = upload(s)) != ZT_OK) return rc;
  RenderParams p = make_params(s, o);
  p.row0 = row_begin;
  p.rows = row_end - row_begin;
  const uint32_t n_params = (uint32_t)(s->materials.size() * 3);
  memset(d_colors, 0, n_params * sizeof(double));
  if (p.max_depth == 0 || n_params == 0) return ZT_OK;
  const std::vector<double> th = theta_host(s, colors);
  const zt_diff_cache& cache = s->device->diff;
  const bool cached = cache.valid && same_render(cache.opts, *o) && cache.theta == th && cache.row0 <= p.row0 &&
                      p.row0 + p.rows <= cache.row0 + cache.rows &&
                      memcmp(&cache.camera, &s->camera, sizeof s->camera) == 0 &&
                      memcmp(&cache.background, &s->background, sizeof s->background) == 0;
  const double* sample_L = cached ? cache.L : nullptr;
  const size_t img_bytes = (size_t)(p.rows * o->width * 3) * sizeof(double);
  double *d_theta = nullptr, *d_img = nullptr, *d_grad = nullptr;
  if ((rc = upload_theta(th, &d_theta)) != ZT_OK) return rc;
  rc = pool_alloc((void**)&d_img, img_bytes, 0, "allocate image adjoint");
  if (rc == ZT_OK) rc = pool_alloc((void**)&d_grad, n_params * sizeof(double), 0, "allocate gradients");
  if (rc != ZT_OK) {
    pool_free(d_theta, 0);
    pool_free(d_img, 0);
    return rc;
  }
  cudaError_t e = cudaMemcpy(d_img, d_image, img_bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d_grad, 0, n_params * sizeof(double));
  if (e == cudaSuccess) e = cudaMemsetAsync(s->device->counter, 0, sizeof(unsigned int), 0);
  if (e == cudaSuccess) {
    const size_t smem = (size_t)n_params * sizeof(double) * (128 / 32); /* one slice per warp */
    const int use_smem = smem <= 48 * 1024 ? 1 : 0;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_backward_diff<128>, 128, use_smem ? smem : 0);
    uint64_t blocks = (uint64_t)sm_count() * (per_sm > 0 ? per_sm : 1);
    const uint64_t need = (p.width * p.rows + 127) / 128;
    if (blocks > need) blocks = need;
    k_backward_diff<128><<<(unsigned)blocks, 128, use_smem ? smem : 0>>>(
        launch_view(s), p, d_theta, d_img, d_grad, n_params, use_smem, sample_L, s->device->counter);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(d_colors, d_grad, n_params * sizeof(double), cudaMemcpyDeviceToHost);
  pool_free(d_theta, 0);
  pool_free(d_img, 0);
  pool_free(d_grad, 0);
  if (e != cudaSuccess) return cuda_fail(e, "zt_backward");
  return ZT_OK;
}

}  /* extern "C" */

/* --------------------------------------------------------- Batched form ---- */
/* A prepared batch: the items table on the device and an executable graph
 * holding [reset counter, one persistent k_render_batch launch]. */
struct zt_batch {
  int device = -1;
  uint64_t n = 0;
  uint64_t total_tiles = 0;
  uint32_t block_size = 128;
  bool nee = true; /* some render of the batch samples lights */
  bool fast = false; /* every render takes the fast traversal */
  bool regen = false; /* the path-regeneration form of the batched kernel */
  BatchItem* d_items = nullptr;
  unsigned int* d_counter = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace zt {

template <int BS, bool kNee, bool kFast>
static void launch_batch_kernel(const zt_batch* b, cudaStream_t st) {
  k_render_batch<BS, kNee, kFast>
      <<<persistent_grid(k_render_batch<BS, kNee, kFast>, BS, b->total_tiles * 32), BS, 0, st>>>(
          b->d_items, (uint32_t)b->n, b->total_tiles, b->d_counter);
}

template <int BS, bool kFast>
static void launch_batch_regen(const zt_batch* b, cudaStream_t st) {
  k_render_batch_regen<BS, kFast>
      <<<persistent_grid(k_render_batch_regen<BS, kFast>, BS, b->total_tiles * 32), BS, 0, st>>>(
          b->d_items, (uint32_t)b->n, b->total_tiles, b->d_counter);
}

template <int BS>
static void launch_batch_bs(const zt_batch* b, cudaStream_t st) {
  if (b->regen) {
    if (b->fast) launch_batch_regen<BS, true>(b, st);
    else launch_batch_regen<BS, false>(b, st);
    return;
  }
  if (b->fast) {
    if (b->nee) launch_batch_kernel<BS, true, true>(b, st);
    else launch_batch_kernel<BS, false, true>(b, st);
  } else {
    if (b->nee) launch_batch_kernel<BS, true, false>(b, st);
    else launch_batch_kernel<BS, false, false>(b, st);
  }
}

static void batch_free(zt_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  cudaFree(b->d_items);
  cudaFree(b->d_counter);
  delete b;
}

}  // namespace zt

extern "C" {

zt_status zt_batch_create(zt_scene* const* scenes, const zt_options* opts, uint64_t n, double* const* d_outs,
                          const zt_gpu_config* cfg, uint32_t order, zt_batch** out) {
  if (!scenes || !opts || !d_outs || !out || n == 0 || n > 0xFFFFFFFFull)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_batch_create: NULL argument or empty batch");
  *out = nullptr;
  const uint32_t bs = cfg ? cfg->block_size : 0;
  if (!valid_block_size(bs)) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_gpu_config.block_size must be 0, 64, 128 or 256");
  if (order > 1) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_batch_create: order must be 0 (as given) or 1 (largest first)");
  const uint32_t bmode = cfg ? cfg->mode : ZT_MODE_AUTO;
  if (bmode != ZT_MODE_AUTO && bmode != ZT_MODE_MEGAKERNEL && bmode != ZT_MODE_MEGAKERNEL_REGEN)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_batch_create: a batch runs the megakernel (mode 0 or 1) or its "
                                         "path-regeneration form (mode 3)");
  std::vector<uint64_t> idx(n);
  std::vector<double> cost(n);
  for (uint64_t i = 0; i < n; ++i) {
    zt_status rc = check_render_args(scenes[i], &opts[i]);
    if (rc != ZT_OK) return rc;
    if (!d_outs[i]) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_batch_create: NULL output");
    rc = upload(scenes[i], false); /* copies in flight; one synchronisation below */
    if (rc != ZT_OK) return rc;
    idx[i] = i;
    /* expected work: samples x log2 of the primitive count */
    cost[i] = (double)(opts[i].width * opts[i].height * opts[i].spp) *
              log2((double)scenes[i]->shapes.size() + scenes[i]->planes.size() + 2.0);
  }
  ZT_CUDA(cudaStreamSynchronize(0), "upload the batch's scenes");
  if (order == 1) std::stable_sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return cost[a] > cost[b]; });
  std::vector<BatchItem> items(n);
  uint64_t tiles = 0;
  for (uint64_t k = 0; k < n; ++k) {
    const uint64_t i = idx[k];
    BatchItem& it = items[k];
    it.sc = launch_view(scenes[i]);
    it.p = make_params(scenes[i], &opts[i]);
    it.out = d_outs[i];
    it.tiles_x = (opts[i].width + 7) / 8;
    it.tile_begin = tiles;
    tiles += it.tiles_x * ((opts[i].height + 3) / 4);
  }
  if (tiles >= (1ull << 32)) return fail(ZT_ERR_INVALID_OPTIONS, "zt_batch_create: more than 2^32 tiles in the batch");
  for (uint64_t k = 0; k < n; ++k)
    if (items[k].p.max_depth == 0)
      return fail(ZT_ERR_INVALID_OPTIONS, "zt_batch_create: max_depth 0 renders are all zero; render them alone");
  zt_batch* b = new (std::nothrow) zt_batch();
  if (!b) return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory");
  b->n = n;
  b->total_tiles = tiles;
  b->block_size = bs ? bs : 128;
  b->nee = false;
  for (uint64_t k = 0; k < n; ++k) b->nee = b->nee || items[k].p.use_nee != 0;
  const uint32_t precision = cfg ? cfg->precision : ZT_PRECISION_EXACT;
  if (precision > ZT_PRECISION_FAST) {
    delete b;
    return fail(ZT_ERR_INVALID_ARGUMENT, "unknown zt_gpu_config.precision");
  }
  b->fast = precision == ZT_PRECISION_FAST;
  b->regen = bmode == ZT_MODE_MEGAKERNEL_REGEN;
  for (uint64_t k = 0; k < n && b->fast; ++k) b->fast = use_fast(scenes[idx[k]], items[k].p, precision, false);
  cudaError_t e = cudaGetDevice(&b->device);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_items, n * sizeof(BatchItem));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_counter, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemcpy(b->d_items, items.data(), n * sizeof(BatchItem), cudaMemcpyHostToDevice);
  cudaStream_t cs = nullptr;
  cudaGraph_t g = nullptr;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned int), cs);
    if (b->block_size == 64) launch_batch_bs<64>(b, cs);
    else if (b->block_size == 256) launch_batch_bs<256>(b, cs);
    else launch_batch_bs<128>(b, cs);
    const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
    e = e2 != cudaSuccess ? e2 : cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
  if (g) cudaGraphDestroy(g);
  if (cs) cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    batch_free(b);
    return cuda_fail(e, "zt_batch_create");
  }
  *out = b;
  return ZT_OK;
}

zt_status zt_batch_launch(zt_batch* b, void* stream) {
  if (!b) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_batch_launch: NULL batch");
  ZT_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream), "zt_batch_launch");
  return ZT_OK;
}

void zt_batch_destroy(zt_batch* b) { batch_free(b); }

zt_status zt_render_batch(zt_scene* const* scenes, const zt_options* opts, uint64_t n, double* const* outs,
                          const zt_gpu_config* cfg) {
  if (!scenes || !opts || !outs || n == 0) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_batch: NULL argument");
  std::vector<size_t> off(n + 1, 0);
  for (uint64_t i = 0; i < n; ++i) {
    if (!opts[i].width || !opts[i].height) return fail(ZT_ERR_INVALID_OPTIONS, "InvalidOptions");
    off[i + 1] = off[i] + (size_t)(opts[i].width * opts[i].height * 3);
  }
  double* d = nullptr;
  zt_status rc = pool_alloc((void**)&d, off[n] * sizeof(double), 0, "allocate batch framebuffers");
  if (rc != ZT_OK) return rc;
  std::vector<double*> d_outs(n);
  for (uint64_t i = 0; i < n; ++i) d_outs[i] = d + off[i];
  zt_batch* b = nullptr;
  rc = zt_batch_create(scenes, opts, n, d_outs.data(), cfg, 1, &b);
  if (rc == ZT_OK) rc = zt_batch_launch(b, nullptr);
  if (rc == ZT_OK) { /* every image back, then one synchronisation */
    cudaError_t e = cudaSuccess;
    for (uint64_t i = 0; i < n && e == cudaSuccess; ++i)
      e = cudaMemcpyAsync(outs[i], d_outs[i], (off[i + 1] - off[i]) * sizeof(double), cudaMemcpyDeviceToHost, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) rc = cuda_fail(e, "copy batch framebuffers");
  }
  zt_batch_destroy(b);
  pool_free(d, 0);
  return rc;
}

}  /* extern "C" */

/* ----------------------------------------------- Allocation-free render ---- */
/*
 * zt_render_noalloc is for callers that must not allocate device memory once
 * they are rendering: an engine or service that hands every byte of the GPU
 * to its own pool at start-up and forbids allocations afterwards, or a
 * real-time loop that cannot afford the allocator's synchronisation.  The
 * scene is uploaded once at
 * set-up (zt_scene_upload allocates; do it before the loop).  Per call, the
 * only device memory used beyond the uploaded scene is the scratch below:
 * the persistent grid's work counter and a staging framebuffer for at most
 * ZT_NOALLOC_MAX_PIXELS pixels, copied into the caller's host buffer.
 *
 * The array is a file-scope __device__ object: every GPU that loads this
 * library holds its 6 MiB until the process exits.  All calls share it and it
 * keeps the last call's contents; the counter is cleared at the start of each
 * call.  Calls whose GPU work overlaps (different streams or threads at the
 * same time) race on it.
 */
static __device__ __align__(256) unsigned char g_noalloc_scratch[ZT_NOALLOC_FB_OFFSET +
                                                                 (size_t)ZT_NOALLOC_MAX_PIXELS * 3 * sizeof(double)];

namespace zt {

/* The megakernel writing into the static scratch (counter at offset 0,
 * framebuffer at ZT_NOALLOC_FB_OFFSET). */
__global__ void __launch_bounds__(128, 7) k_render_mega_noalloc(DevScene sc, RenderParams p,
                                                                unsigned char* __restrict__ scratch) {
  unsigned int* counter = reinterpret_cast<unsigned int*>(scratch);
  double* out = reinterpret_cast<double*>(scratch + ZT_NOALLOC_FB_OFFSET);
  const uint64_t tiles_x = (p.width + 7) / 8, tiles = tiles_x * ((p.height + 3) / 4);
  const unsigned lane = threadIdx.x & 31;
  for (;;) {
    unsigned tile = 0;
    if (lane == 0) tile = atomicAdd(counter, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if ((uint64_t)tile >= tiles) return;
    const uint64_t x = (tile % tiles_x) * 8 + (lane & 7), y = (tile / tiles_x) * 4 + (lane >> 3);
    if (x < p.width && y < p.height) render_pixel<false>(sc, p, y * p.width + x, out, nullptr);
  }
}

/* In host code g_noalloc_scratch names a host-side stand-in, not device
 * memory: its device address is looked up once per device, with that device
 * current, and cached.  The lookup may load this library's GPU code on that
 * device, which is why the first call on a device belongs before any stream
 * capture.  The address belongs to the device's context: after a
 * cudaDeviceReset the module is loaded again, possibly elsewhere, so each
 * cached address carries the unique id of the context it was looked up in
 * (cuCtxGetId, reached through the runtime's driver entry point) and is
 * looked up again when the current context's id differs. */
static std::mutex g_noalloc_mutex;
static unsigned char* g_noalloc_ptr[256] = {};
static unsigned long long g_noalloc_ctx[256] = {};

typedef int (*ZtCtxGetCurrent)(void** ctx);
typedef int (*ZtCtxGetId)(void* ctx, unsigned long long* id);

/* Id of the current context, 0 when the driver cannot tell. */
static unsigned long long current_context_id() {
  static ZtCtxGetCurrent get_current = nullptr;
  static ZtCtxGetId get_id = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    looked_up = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<ZtCtxGetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<ZtCtxGetId>(f);
    cudaGetLastError();
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

static zt_status noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= 256) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  const unsigned long long ctx = current_context_id();
  if (!g_noalloc_ptr[dev] || ctx != g_noalloc_ctx[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
    g_noalloc_ctx[dev] = ctx;
  }
  *out = g_noalloc_ptr[dev];
  return ZT_OK;
}

}  // namespace zt

extern "C" zt_status zt_render_noalloc(zt_scene* s, const zt_options* o, double* out_rgb, void* stream) {
  zt_status rc = check_render_args(s, o);
  if (rc != ZT_OK) return rc;
  if (!out_rgb) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_noalloc: NULL output");
  const uint64_t npix = o->width * o->height;
  if (npix > ZT_NOALLOC_MAX_PIXELS)
    return fail(ZT_ERR_INVALID_ARGUMENT, "zt_render_noalloc: " + std::to_string(o->width) + "x" +
                                             std::to_string(o->height) + " is " + std::to_string(npix) +
                                             " pixels, more than its static scratch holds (maximum " +
                                             std::to_string(ZT_NOALLOC_MAX_PIXELS) + " pixels)");
  int dev = 0;
  ZT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (!s->device || s->device->device != dev)
    return fail(ZT_ERR_INVALID_ARGUMENT,
                "zt_render_noalloc: scene is not resident on the current device; call zt_scene_upload at set-up");
  unsigned char* scratch = nullptr;
  rc = noalloc_scratch(dev, &scratch);
  if (rc != ZT_OK) return rc;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const RenderParams p = make_params(s, o);
  double* fb = reinterpret_cast<double*>(scratch + ZT_NOALLOC_FB_OFFSET);
  const size_t bytes = (size_t)npix * 3 * sizeof(double);
  if (p.max_depth == 0) { /* traceWith never enters its loop: every sample is zero */
    ZT_CUDA(cudaMemsetAsync(fb, 0, bytes, st), "clear framebuffer");
  } else {
    ZT_CUDA(cudaMemsetAsync(scratch, 0, sizeof(unsigned int), st), "clear work counter");
    k_render_mega_noalloc<<<persistent_grid(k_render_mega_noalloc, 128, npix), 128, 0, st>>>(launch_view(s), p,
                                                                                          scratch);
    ZT_CUDA(cudaGetLastError(), "launch k_render_mega_noalloc");
  }
  ZT_CUDA(cudaMemcpyAsync(out_rgb, fb, bytes, cudaMemcpyDeviceToHost, st), "copy framebuffer");
  ZT_CUDA(cudaStreamSynchronize(st), "zt_render_noalloc");
  return ZT_OK;
}

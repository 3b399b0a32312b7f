/*
 * zigtrace_b200.h -- C ABI of the B200 (sm_100a) renderer for zigtrace's
 * per-pixel radiance path.
 *
 * This is the drop-in boundary for avohra25/zigtrace's library API
 * (src/root.zig:2-17): scene construction (src/scene.zig:53-96), rendering
 * to an f64 HDR framebuffer (src/render.zig:152-180) and the 8-bit encode
 * (src/image.zig:24-73).  Every entry point is `extern "C"`, takes plain
 * pointers and sizes, and blocks until its result is in the caller's buffer
 * unless it says otherwise.  All arithmetic on the path is IEEE f64 without
 * FMA contraction, as in the reference, so images are bit-identical to the
 * reference algorithm's for the same scene, options and seed.
 *
 * Errors: every call returns a zt_status; on failure zt_last_error() returns
 * a message for the calling thread.  Status values map onto the reference's
 * Zig error set as noted.
 */
#ifndef ZIGTRACE_B200_H
#define ZIGTRACE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t zt_status;
#define ZT_OK 0
#define ZT_ERR_INVALID_OPTIONS (-1)     /* error.InvalidOptions, src/render.zig:153 */
#define ZT_ERR_OUT_OF_MEMORY (-2)       /* error.OutOfMemory (host or device) */
#define ZT_ERR_TOO_MANY_PRIMITIVES (-3) /* error.TooManyPrimitives, src/bvh.zig:44 */
#define ZT_ERR_UNBOUNDED_SHAPE (-4)     /* error.UnboundedShape, src/bvh.zig:55 */
#define ZT_ERR_INVALID_ARGUMENT (-5)    /* bad pointer, index or enum value */
#define ZT_ERR_CUDA (-6)                /* a CUDA runtime call failed */
#define ZT_ERR_TIMEOUT (-7)             /* a bounded device wait gave up */
#define ZT_ERR_NOT_BUILT (-8)           /* render before zt_scene_build */

typedef struct { double x, y, z; } zt_vec3; /* Vec3, src/vec.zig:5-8 */

/* Shape, src/geometry.zig:229-248.  p[] holds
 *   ZT_SPHERE:   center.xyz, radius (negative radius = inward normals)
 *   ZT_TRIANGLE: v0.xyz, v1.xyz, v2.xyz
 *   ZT_PLANE:    point.xyz, unit normal.xyz                                   */
enum { ZT_SPHERE = 0, ZT_TRIANGLE = 1, ZT_PLANE = 2 };
typedef struct { uint32_t kind; uint32_t material; double p[9]; } zt_shape;

/* Material, src/material.zig:15-24.  color is the albedo (lambertian,
 * metal) or the emitted radiance (emissive); param is the metal fuzz or the
 * dielectric index of refraction. */
enum { ZT_LAMBERTIAN = 0, ZT_METAL = 1, ZT_DIELECTRIC = 2, ZT_EMISSIVE = 3 };
typedef struct { uint32_t kind; uint32_t reserved; zt_vec3 color; double param; } zt_material;

/* CameraConfig, src/camera.zig:8-18; focus_dist is used when
 * has_focus_dist != 0, else |look_from - look_at|. */
typedef struct {
  zt_vec3 look_from, look_at, up;
  double vfov, aperture, focus_dist;
  uint32_t has_focus_dist, reserved;
} zt_camera_config;

/* Background, src/scene.zig:15-28: ZT_BG_SOLID uses a; ZT_BG_SKY blends from
 * horizon a to zenith b. */
enum { ZT_BG_SOLID = 0, ZT_BG_SKY = 1 };
typedef struct { uint32_t kind; uint32_t reserved; zt_vec3 a, b; } zt_background;

/* render.Options, src/render.zig:12-23.  threads and tile_size keep their
 * reference meaning for validation (tile_size == 0 is InvalidOptions); the
 * device schedules its own work. */
typedef struct {
  uint64_t width, height, spp, max_depth, threads, seed, tile_size;
  uint32_t light_sampling, reserved;
} zt_options;

/* Bvh.Node, src/bvh.zig:22-33 (host copy, for inspection). */
typedef struct { zt_vec3 bmin, bmax; uint32_t first, count; } zt_bvh_node;
/* Light, src/light.zig:30-35 (host copy, for inspection). */
typedef struct { zt_shape shape; zt_vec3 radiance; double weight; } zt_light;

/* Device-side execution choices; zero-initialised means "defaults".
 * MEGAKERNEL: one persistent kernel, each warp renders an 8x4 pixel tile
 * sample by sample.  WAVEFRONT: per-bounce kernels over ray queues in a CUDA
 * graph.  MEGAKERNEL_REGEN: the megakernel with per-lane path regeneration
 * (a lane whose path ends starts its next sample at once); faster on closed
 * scenes with long paths.  AUTO is MEGAKERNEL_REGEN when the mean path
 * length of a 64x64, 1-spp pilot traced at zt_scene_upload is at least 3,
 * else MEGAKERNEL.  WAVEFRONT_SORTED: the wavefront form with its extension
 * queue sorted between bounces by ray direction octant and origin cell.
 * All modes give bit-identical images. */
enum { ZT_MODE_AUTO = 0, ZT_MODE_MEGAKERNEL = 1, ZT_MODE_WAVEFRONT = 2, ZT_MODE_MEGAKERNEL_REGEN = 3,
       ZT_MODE_WAVEFRONT_SORTED = 4 };
/* ZT_PRECISION_EXACT (the default) is the verification build of the path:
 * every operation is the reference's f64 operation in the reference's order,
 * so images are bit-identical to the reference algorithm's as restated by
 * the project's CPU oracle (which shares this library's sin/cos, so parity
 * with Zig's own transcendentals is not covered).
 * ZT_PRECISION_FAST tests BVH boxes in single precision against conservative
 * (outward-rounded, widened) copies of the f64 boxes; primitive tests, hit
 * records and shading stay the reference's f64 operations.  It visits every
 * BVH leaf the exact walk visits (and some more), so the closest hit differs
 * only on exact ties and rays that graze a box edge: images agree with the
 * exact ones to far below Monte Carlo noise, though not bit for bit.  Used by
 * the megakernel modes and the batch; single renders of scenes with fewer
 * than 64 bounded primitives (where the float walk does not pay), and any
 * render whose scene has leaves of more than 15 primitives or bounds or a
 * camera beyond 1e7 in magnitude, render exact (a batch takes the fast walk
 * only if all of its renders can). */
enum { ZT_PRECISION_EXACT = 0, ZT_PRECISION_FAST = 1 };
typedef struct {
  uint32_t mode;           /* ZT_MODE_* */
  uint32_t block_size;     /* threads per block, 0 = default */
  uint32_t queue_capacity; /* wavefront: paths in flight, 0 = default */
  uint32_t precision;      /* ZT_PRECISION_* */
} zt_gpu_config;

typedef struct zt_scene zt_scene;

/* ---- Scene construction (src/scene.zig:53-96) ------------------------- */
/* Scene.init: an empty scene with the reference defaults (camera from the
 * origin looking down -z, vfov 60; sky background 1,1,1 -> 0.5,0.7,1.0). */
zt_status zt_scene_create(zt_scene** out);
void zt_scene_destroy(zt_scene* scene);
/* Scene.addMaterial; writes the new material id. */
zt_status zt_scene_add_material(zt_scene* scene, const zt_material* m, uint32_t* id_out);
/* Scene.addMaterial for n materials; writes the id of the first one. */
zt_status zt_scene_add_materials(zt_scene* scene, const zt_material* m, size_t n, uint32_t* first_id_out);
/* Scene.add for n shapes; planes go to the unbounded list (scene.zig:71-78).
 * Invalidates a previous build. */
zt_status zt_scene_add_shapes(zt_scene* scene, const zt_shape* shapes, size_t n);
/* Scene.addQuad: corner + a*u + b*v as two triangles (scene.zig:82-88). */
zt_status zt_scene_add_quad(zt_scene* scene, const zt_vec3* corner, const zt_vec3* u,
                            const zt_vec3* v, uint32_t material);
zt_status zt_scene_set_camera(zt_scene* scene, const zt_camera_config* cfg);
zt_status zt_scene_set_background(zt_scene* scene, const zt_background* bg);
/* Scene.build: binned-SAH BVH and the emitter table, on the host
 * (bvh.zig:41-67, light.zig:68-94). */
zt_status zt_scene_build(zt_scene* scene);
/* Scene.build with the BVH built on the current CUDA device: the same nodes,
 * primitive order and numbering as zt_scene_build (bvh.zig:41-262), node
 * bounds equal up to the sign of zero.  Scenes that need the reference's
 * median split (more than 4 primitives whose centroids coincide, or bounds
 * without area) or hold non-finite coordinates are built on the host, as are
 * all scenes when no CUDA device (or too little device memory) is available;
 * *used_device (may be NULL) is 1 when the device built the BVH.
 * *build_ms (may be NULL) is the device time of the build. */
zt_status zt_scene_build_device(zt_scene* scene, uint32_t* used_device, double* build_ms);

/* Scene.build with the BVH the caller already built: the reference's
 * Bvh.build output (bvh.zig:41-67; Node at bvh.zig:22-33, the shape
 * permutation at bvh.zig:35-38), passed as n_nodes nodes and n_indices
 * shape indices (n_indices = number of bounded shapes), used as given
 * without rebuilding.  The emitter table is built as Scene.build does
 * (light.zig:68-94).  The tree must be one the reference's build can
 * produce in shape: root at 0, each interior node's two children adjacent at
 * an odd index after it, every node reachable once, depth at most 64, leaves
 * covering every shape position once, indices a permutation; anything else
 * is ZT_ERR_INVALID_ARGUMENT and leaves the scene unbuilt. */
zt_status zt_scene_set_bvh(zt_scene* scene, const zt_bvh_node* nodes, size_t n_nodes, const uint32_t* indices,
                           size_t n_indices);

/* ---- Inspection (Scene fields, Bvh, Lights) --------------------------- */
zt_status zt_scene_counts(const zt_scene* scene, uint64_t* n_materials, uint64_t* n_bounded,
                          uint64_t* n_planes, uint64_t* n_nodes, uint64_t* n_lights);
zt_status zt_scene_bvh(const zt_scene* scene, zt_bvh_node* nodes_out, uint32_t* indices_out);
zt_status zt_scene_lights(const zt_scene* scene, zt_light* lights_out, double* cdf_out,
                          double* total_out);
zt_status zt_scene_bvh_depth(const zt_scene* scene, uint64_t* depth_out);

/* ---- Device residency -------------------------------------------------- */
/* Copies the built scene to the current CUDA device (kept until the scene is
 * changed, destroyed, or zt_scene_release_device is called). */
zt_status zt_scene_upload(zt_scene* scene);
zt_status zt_scene_release_device(zt_scene* scene);
/* Bytes one upload copies host-to-device (the flattened scene is kept in
 * pinned host memory after the first upload, so re-uploads are one copy). */
zt_status zt_scene_upload_bytes(zt_scene* scene, uint64_t* bytes);

/* ---- Rendering (src/render.zig:152-180) -------------------------------- */
/* render.render into a caller-owned host buffer of width*height*3 doubles,
 * row-major, top row first.  Uploads the scene if it is not resident. */
zt_status zt_render(zt_scene* scene, const zt_options* opts, double* out_rgb);
/* render.render restricted to image rows [row_begin, row_end) of the
 * width x height image: same camera, same per-pixel RNG streams, so the band
 * equals those rows of zt_render's image.  Used to shard one image across
 * devices (each renders a band; the bands are gathered).  out has
 * (row_end - row_begin)*width*3 doubles. */
zt_status zt_render_rows(zt_scene* scene, const zt_options* opts, uint64_t row_begin, uint64_t row_end,
                         double* out_rgb);
/* The same with explicit device choices (cfg may be NULL). */
zt_status zt_render_ex(zt_scene* scene, const zt_options* opts, const zt_gpu_config* cfg,
                       double* out_rgb);
/* Device-resident form: d_out_rgb is a device pointer (width*height*3
 * doubles); the work is enqueued on `stream` (a cudaStream_t, NULL = legacy
 * default stream) and the call returns without synchronising.  The scene
 * must have been uploaded to the current device. */
zt_status zt_render_device(zt_scene* scene, const zt_options* opts, const zt_gpu_config* cfg,
                           double* d_out_rgb, void* stream);
/* Upper bound on the iterations of the wavefront loop, which runs on the
 * device (a CUDA-graph while node): a render that reaches it stops and its
 * zt_render / zt_render_ex call returns ZT_ERR_TIMEOUT.  The default (0)
 * bound is pixels x spp x (max_depth + 1), which no correct render reaches;
 * a lower one makes the bound fire, to exercise that error path.
 * Process-wide. */
zt_status zt_set_wavefront_iteration_limit(uint64_t max_iterations);
/* Device-resident band: rows [row_begin, row_end) of the width x height
 * image (the same camera and per-pixel RNG streams, so the band equals those
 * rows of the whole image) into the device buffer d_out_rgb of
 * (row_end - row_begin)*width*3 doubles, enqueued on `stream` without
 * synchronising.  One rank's share of a frame sharded across GPUs, written
 * straight into its slot of a collective's buffer.  Megakernel modes only
 * (ZT_MODE_WAVEFRONT is rejected); cfg may be NULL.  The scene must have been
 * uploaded to the current device. */
zt_status zt_render_rows_device(zt_scene* scene, const zt_options* opts, uint64_t row_begin, uint64_t row_end,
                                const zt_gpu_config* cfg, double* d_out_rgb, void* stream);
/* ---- Differentiable form ------------------------------------------------ */
/* Gradients of an image loss with respect to every material's colour (the
 * albedo of Lambertian and metal materials, the radiance of emissive ones;
 * colors[3*m + c]).  Sampling is detached: the scene's own materials drive
 * every sampling decision (roulette, light pick, MIS weights), `colors` (NULL
 * = the scene's own) only the contributions, so with common random numbers
 * the image is a smooth function of `colors`; with colors == NULL it is
 * zt_render's image.  zt_forward renders into out_rgb (width*height*3);
 * zt_backward takes dL/dimage (width*height*3) and writes dL/dcolors
 * (n_materials*3), replaying each path from its RNG stream (no tape).
 * Gradients are accumulated with atomics, so their last bits may vary
 * between runs.
 * Memory: zt_forward keeps every sample's primal radiance on the device for
 * the next zt_backward with the same options, colours, camera and
 * background (24 bytes per sample of the whole image: 403 MB at 512x512x64)
 * when that fits the scene's primal cache limit (default 1 GiB); above the
 * limit nothing is kept and zt_backward traces the primal itself, which
 * gives the same gradients. */
zt_status zt_forward(zt_scene* scene, const zt_options* opts, const double* colors, double* out_rgb);
zt_status zt_backward(zt_scene* scene, const zt_options* opts, const double* colors, const double* d_image,
                      double* d_colors);
/* Largest primal cache (bytes) zt_forward may keep for this scene; 0 keeps
 * none.  Lowering it below the cache held now frees that cache. */
zt_status zt_scene_set_primal_cache_limit(zt_scene* scene, uint64_t max_bytes);
/* The same for the image rows [row_begin, row_end) (one band of a frame
 * sharded across GPUs): out_rgb and d_image hold the band's rows only,
 * d_colors the band's share of the gradient (the shares of all bands sum to
 * zt_backward's).  A zt_backward_rows after a zt_forward_rows over a band
 * containing its rows, with the same options and colours, reuses the
 * forward's primal radiance. */
zt_status zt_forward_rows(zt_scene* scene, const zt_options* opts, uint64_t row_begin, uint64_t row_end,
                          const double* colors, double* out_rgb);
zt_status zt_backward_rows(zt_scene* scene, const zt_options* opts, uint64_t row_begin, uint64_t row_end,
                           const double* colors, const double* d_image, double* d_colors);

/* ---- Batched form: many renders in one persistent launch --------------- */
/* n renders (scenes[i] with opts[i] into the device buffer d_outs[i] of
 * width*height*3 doubles) prepared as one persistent kernel launch captured
 * in a CUDA graph.  Every pixel equals what zt_render gives for that scene
 * and those options.  order: 0 = tiles in the given order, 1 = largest
 * renders first.  Scenes are uploaded to the current device if needed.  The
 * batch keeps pointers to the scenes' device copies: destroy it before the
 * scenes change or are destroyed.  block_size in cfg: 0/64/128/256; mode:
 * ZT_MODE_AUTO or ZT_MODE_MEGAKERNEL (the nested megakernel) or
 * ZT_MODE_MEGAKERNEL_REGEN (per-lane path regeneration); precision as for a
 * single render. */
typedef struct zt_batch zt_batch;
zt_status zt_batch_create(zt_scene* const* scenes, const zt_options* opts, uint64_t n, double* const* d_outs,
                          const zt_gpu_config* cfg, uint32_t order, zt_batch** out);
/* Replays the batch's graph on `stream` (a cudaStream_t) without waiting. */
zt_status zt_batch_launch(zt_batch* batch, void* stream);
void zt_batch_destroy(zt_batch* batch);
/* Convenience: the batch into host buffers outs[i] (blocking). */
zt_status zt_render_batch(zt_scene* const* scenes, const zt_options* opts, uint64_t n, double* const* outs,
                          const zt_gpu_config* cfg);

/* Allocation-free render, for callers that must not allocate device memory
 * while rendering: an engine or service that hands the GPU's memory to its
 * own pool at start-up and fails or stalls on any allocation made behind its
 * back afterwards, or a frame loop that cannot afford the device-wide
 * synchronisation a cudaMalloc/cudaFree pair can cost.  It has no
 * counterpart in the reference.  The scene must already be resident
 * (zt_scene_upload, which allocates, belongs at set-up).  The call uses no memory beyond the scene but
 * a 6 MiB scratch array compiled into the library (held by every GPU that
 * loads it, for the life of the process): the work counter and a staging
 * framebuffer of at most ZT_NOALLOC_MAX_PIXELS pixels; larger images are
 * rejected with ZT_ERR_INVALID_ARGUMENT.  The result is written to the
 * caller's host buffer (width*height*3 doubles) and the call returns after
 * synchronising `stream` (a cudaStream_t, NULL = legacy default stream).
 * The first call on a device looks up the scratch's device address (and may
 * load the library's GPU code there): make it before any stream capture.
 * The address is looked up again when the device's context changes (after
 * cudaDeviceReset, for instance).  All calls share the scratch and it keeps
 * the last call's contents, so calls whose GPU work overlaps race. */
#define ZT_NOALLOC_MAX_PIXELS (512u * 512u)
#define ZT_NOALLOC_FB_OFFSET 256u
zt_status zt_render_noalloc(zt_scene* scene, const zt_options* opts, double* out_rgb, void* stream);
/* First sample of every pixel on the device: primitive id of the camera
 * ray's closest hit (bounded-shape index, or n_bounded + plane index, -1 on a
 * miss) and the number of extension rays the path traced.  Host buffers of
 * width*height entries. */
zt_status zt_render_debug(zt_scene* scene, const zt_options* opts, int32_t* first_prim_out,
                          uint32_t* path_len_out);
/* render.traceWith (src/render.zig:61-102) n times along one ray, drawing
 * every path from one RNG stream in sequence, as the reference's own tests
 * do (meanRadiance, src/render.zig:290-302).  rng_state (4 x u64, the Rng.s
 * words) is read and updated; out has n*3 doubles.  Runs on the device. */
zt_status zt_trace_paths(zt_scene* scene, const zt_vec3* origin, const zt_vec3* dir, uint64_t* rng_state,
                         uint64_t n, uint64_t max_depth, uint32_t light_sampling, double* out);
/* Rng.forStream(seed, stream_index) followed by n_draws Rng.next() on the
 * device, for n_streams consecutive stream indices starting at stream0
 * (src/rng.zig:22-38).  out has n_streams*n_draws entries. */
zt_status zt_rng_streams(uint64_t seed, uint64_t stream0, uint64_t n_streams, uint64_t n_draws,
                         uint64_t* out);

/* ---- Output (src/image.zig:14-73) -------------------------------------- */
/* Image.toRgb8: exposure, tonemap (0 none, 1 reinhard, 2 aces), gamma, round
 * to u8, on the host.  rgb_out has n_pixels*3 bytes. */
zt_status zt_image_to_rgb8(const double* pixels, uint64_t n_pixels, uint32_t tonemap, double gamma,
                           double exposure, uint8_t* rgb_out);
/* Image.toRgb8 on the device: d_pixels (n_pixels*3 f64) and d_rgb_out
 * (n_pixels*3 bytes) are device pointers; asynchronous on `stream` (a
 * cudaStream_t, NULL for the default stream).  The same bytes as
 * zt_image_to_rgb8 except where pow() of the two math libraries rounds a
 * value to opposite sides of a u8 rounding boundary (at most 1 LSB). */
zt_status zt_image_to_rgb8_device(const double* d_pixels, uint64_t n_pixels, uint32_t tonemap, double gamma,
                                  double exposure, uint8_t* d_rgb_out, void* stream);
/* png.writePng (src/png.zig:10-58): the file size for a width x height RGB8
 * image; ZT_ERR_INVALID_ARGUMENT with "InvalidDimensions" (0 or above
 * 2^31-1) or "ImageTooLarge" (zlib stream above 2^31-1 bytes) as the
 * reference reports. */
zt_status zt_png_size(uint64_t width, uint64_t height, uint64_t* bytes_out);
/* png.writePng into a caller buffer of at least zt_png_size bytes: 8-bit
 * RGB, no filtering, stored DEFLATE blocks, on the host. */
zt_status zt_png_encode(const uint8_t* rgb, uint64_t width, uint64_t height, uint8_t* out, uint64_t out_capacity);
/* The same file assembled on the device (d_rgb and d_out device pointers),
 * asynchronous on `stream`; byte-identical to zt_png_encode. */
zt_status zt_png_encode_device(const uint8_t* d_rgb, uint64_t width, uint64_t height, uint8_t* d_out,
                               uint64_t out_capacity, void* stream);
/* render + Image.toRgb8 (the CLI's output path, src/main.zig:243-258) with
 * both stages on the device; only the W*H*3 bytes of rgb_out are copied back.
 * cfg may be NULL. */
zt_status zt_render_rgb8(zt_scene* scene, const zt_options* opts, const zt_gpu_config* cfg, uint32_t tonemap,
                         double gamma, double exposure, uint8_t* rgb_out);
/* render + Image.toRgb8 + png.writePng with every stage on the device; only
 * the PNG file (zt_png_size bytes, png_capacity at least that) is copied
 * back. */
zt_status zt_render_png(zt_scene* scene, const zt_options* opts, const zt_gpu_config* cfg, uint32_t tonemap,
                        double gamma, double exposure, uint8_t* png_out, uint64_t png_capacity);

const char* zt_last_error(void);
/* Library version string. */
const char* zt_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ZIGTRACE_B200_H */

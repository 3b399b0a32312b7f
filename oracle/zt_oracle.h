/*
 * zt_oracle.h -- CPU oracle for the zigtrace radiance path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C, f64, FMA-free restatement of
 * the reference renderer (avohra25/zigtrace, the src/ Zig files) used as the checker
 * for the CUDA path: only the tests, the smoke check and the CPU-baseline leg
 * of the benchmark load it.  The product library never links or calls it.
 *
 * Parity pinning: the reference is Zig 0.14 and no Zig toolchain exists here,
 * so the reference cannot be built or run.  This restatement is pinned by the
 * reference's own known-answer tests (src/render.zig:188-403,
 * src/bvh.zig:316-372, src/light.zig:358-494, src/material.zig:84-142,
 * src/geometry.zig:266-334, src/camera.zig:72-108, src/aabb.zig:92-123,
 * src/vec.zig:129-174, src/rng.zig:92-138, src/image.zig:85-112), restated in
 * tests/test_oracle_kats.py, and by xoshiro256++/SplitMix64 vectors from an
 * independent pure-Python restatement (tests/golden/make_golden.py).  Bit-level
 * parity with Zig's own @sin/@cos and std.math.pow is unpinned: both this
 * oracle and the device use the project's routines in zt_fpmath.h.
 *
 * Data layouts are identical to the product's C-ABI (include/zigtrace_b200.h)
 * so one scene description feeds both.
 */
#ifndef ZT_ORACLE_H
#define ZT_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double x, y, z; } ov3;

enum { O_SPHERE = 0, O_TRIANGLE = 1, O_PLANE = 2 };
enum { O_LAMBERTIAN = 0, O_METAL = 1, O_DIELECTRIC = 2, O_EMISSIVE = 3 };
enum { O_BG_SOLID = 0, O_BG_SKY = 1 };

/* Shape (src/geometry.zig:229-248).  p[] holds sphere {cx,cy,cz,r},
 * triangle {v0,v1,v2} or plane {point, normal}. */
typedef struct { uint32_t kind, material; double p[9]; } oshape;
/* Material (src/material.zig:15-24): color = albedo / emission, param =
 * metal fuzz or dielectric ior. */
typedef struct { uint32_t kind, pad; ov3 color; double param; } omaterial;
/* CameraConfig (src/camera.zig:8-18). */
typedef struct {
  ov3 look_from, look_at, up;
  double vfov, aperture, focus_dist;
  uint32_t has_focus_dist, pad;
} ocamera_config;
/* Background (src/scene.zig:15-28): solid a, or sky horizon a / zenith b. */
typedef struct { uint32_t kind, pad; ov3 a, b; } obackground;
/* render.Options (src/render.zig:12-23). */
typedef struct {
  uint64_t width, height, spp, max_depth, threads, seed, tile_size;
  uint32_t light_sampling, pad;
} ooptions;
/* Bvh.Node (src/bvh.zig:22-33). */
typedef struct { ov3 bmin, bmax; uint32_t first, count; } onode;
/* Camera (src/camera.zig:20-28). */
typedef struct { ov3 origin, upper_left, horizontal, vertical, u, v; double lens_radius; } ocamera;
/* Hit (src/geometry.zig:11-30) plus the primitive id the reference does not
 * carry: index into the bounded shapes, or n_bounded + plane index. */
typedef struct { double t; ov3 point, normal; uint32_t front_face, material; int32_t prim, pad; } ohit;
/* Light (src/light.zig:30-35). */
typedef struct { oshape shape; ov3 radiance; double weight; } olight;

/* Work counters, summed over all samples of a render. */
typedef struct {
  uint64_t samples, ext_rays, shadow_rays, node_pops, slab_tests, sphere_tests, tri_tests,
      plane_tests, hits, nee_samples, pdfhit_calls, pdfhit_light_tests, rng_draws;
} ostats;

typedef struct oscene oscene;

/* Scene.init + add/addMaterial + build (src/scene.zig:53-96). build_bvh = 0
 * leaves the scene unbuilt (brute-force intersection, no lights). Returns 0,
 * -1 invalid argument, -2 out of memory, -3 TooManyPrimitives. */
int ozt_scene_create(const omaterial* mats, size_t n_mats, const oshape* shapes, size_t n_shapes,
                     const ocamera_config* cam, const obackground* bg, int build_bvh, oscene** out);
void ozt_scene_free(oscene* s);
size_t ozt_scene_bounded_count(const oscene* s);
size_t ozt_scene_plane_count(const oscene* s);
size_t ozt_scene_node_count(const oscene* s);
void ozt_scene_nodes(const oscene* s, onode* out);
void ozt_scene_indices(const oscene* s, uint32_t* out);
size_t ozt_scene_light_count(const oscene* s);
void ozt_scene_lights(const oscene* s, olight* out, double* cdf, double* total);
size_t ozt_bvh_depth(const oscene* s);

/* render.render (src/render.zig:152-180): f64 RGB, row-major, top row first.
 * Returns 0 or -1 (error.InvalidOptions). stats may be NULL. */
int ozt_render(const oscene* s, const ooptions* o, double* out_rgb, ostats* stats);
/* The same estimator for a subset of pixels (index y*width+x). */
int ozt_render_pixels(const oscene* s, const ooptions* o, const uint64_t* pixels, size_t n,
                      double* out_rgb, ostats* stats);
/* First sample of every pixel: primitive id of the camera ray's closest hit
 * (-1 on a miss) and the number of extension rays the path traced. */
int ozt_render_debug(const oscene* s, const ooptions* o, int32_t* first_prim, uint32_t* path_len);
/* ozt_render plus, per pixel, the mean over its samples of the squared
 * luminance (0.2126 r + 0.7152 g + 0.0722 b, light.zig:38-40) of each
 * finite sample: the second-moment buffer behind the Monte Carlo standard
 * error of an image's mean luminance. */
int ozt_render_moments(const oscene* s, const ooptions* o, double* out_rgb, double* moments);
/* The same for a list of pixels (as ozt_render_pixels). */
int ozt_render_pixels_moments(const oscene* s, const ooptions* o, const uint64_t* pixels, size_t n,
                              double* out_rgb, double* moments);

/* The differentiable form's forward (detached sampling): the scene's
 * materials drive roulette, light pick and MIS weights, theta (3 per
 * material) the contributions.  theta = the scene's colours gives ozt_render's
 * image.  Single-threaded. */
int ozt_render_params(const oscene* s, const ooptions* o, const double* theta, double* out_rgb);

/* traceWith (src/render.zig:61-102) on one ray with an explicit RNG state. */
void ozt_trace_with(const oscene* s, const ov3* origin, const ov3* dir, uint64_t rng[4],
                    uint64_t max_depth, int light_sampling, ov3* out);
/* Scene.intersect (src/scene.zig:108-116). Returns 1 on hit. */
int ozt_scene_intersect(const oscene* s, const ov3* origin, const ov3* dir, double tmin,
                        double tmax, ohit* out);
int ozt_shape_intersect(const oshape* sh, const ov3* origin, const ov3* dir, double tmin,
                        double tmax, ohit* out);
int ozt_intersect_all(const oshape* shapes, size_t n, const ov3* origin, const ov3* dir,
                      double tmin, double tmax, ohit* out);
/* Lights.sample / pdfHit (src/light.zig:120-198). sample returns 1 when a
 * sample exists and writes dir, distance, radiance, pdf. */
int ozt_lights_sample(const oscene* s, const ov3* origin, uint64_t rng[4], ov3* dir,
                      double* distance, ov3* radiance, double* pdf);
double ozt_lights_pdf_hit(const oscene* s, const ov3* origin, const ohit* hit);
/* Material.emitted / scatter (src/material.zig:26-62). scatter returns 1 and
 * writes attenuation and the scattered ray, or 0 (absorbed). */
void ozt_material_emitted(const omaterial* m, const ohit* hit, ov3* out);
int ozt_material_scatter(const omaterial* m, const ov3* in_origin, const ov3* in_dir,
                         const ohit* hit, uint64_t rng[4], ov3* atten, ov3* out_origin,
                         ov3* out_dir);
double ozt_schlick(double cosine, double eta);
/* Camera.init / ray (src/camera.zig:29-67). */
void ozt_camera_init(const ocamera_config* cfg, double aspect, ocamera* out);
void ozt_camera_ray(const ocamera* cam, double s, double t, uint64_t rng[4], ov3* origin, ov3* dir);
void ozt_background_radiance(const obackground* bg, const ov3* dir, ov3* out);
/* Rng (src/rng.zig:13-88). */
void ozt_rng_init(uint64_t seed, uint64_t out[4]);
void ozt_rng_for_stream(uint64_t seed, uint64_t stream, uint64_t out[4]);
void ozt_rng_next_n(uint64_t rng[4], size_t n, uint64_t* out);
void ozt_rng_float_n(uint64_t rng[4], size_t n, double* out);
uint64_t ozt_rng_below(uint64_t rng[4], uint64_t n);
void ozt_rng_unit_vector(uint64_t rng[4], ov3* out);
void ozt_rng_in_unit_sphere(uint64_t rng[4], ov3* out);
void ozt_rng_in_unit_disk(uint64_t rng[4], ov3* out);
/* Aabb.hit (src/aabb.zig:68-83). Returns 1 and the entry distance. */
int ozt_aabb_hit(const ov3* bmin, const ov3* bmax, const ov3* origin, const ov3* dir,
                 double tmin, double tmax, double* t);
/* Output.encode / Tonemap.apply (src/image.zig:14-37), kind 0 none,
 * 1 reinhard, 2 aces. */
double ozt_tonemap(int kind, double c);
uint8_t ozt_encode(int kind, double gamma, double exposure, double linear);
/* The project's sin/cos/pow5 (zt_fpmath.h), exported for accuracy tests. */
void ozt_sincos(double x, double* s, double* c);
double ozt_pow5(double x);

#ifdef __cplusplus
}
#endif
#endif

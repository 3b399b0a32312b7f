/*
 * zt_oracle.c -- CPU oracle (test infrastructure only; see zt_oracle.h).
 *
 * A line-by-line f64 restatement of avohra25/zigtrace's radiance path.  Every
 * function cites the reference file:line it follows.  Build with
 * -ffp-contract=off and without fast-math so each expression rounds exactly as
 * the reference's strict-float Zig code does; expression order is kept as the
 * reference writes it (e.g. Vec3.div multiplies by the reciprocal).
 */
#define _GNU_SOURCE
#include "zt_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>

#include "zt_fpmath.h"

#define PI 3.14159265358979323846

/* ---------------------------------------------------------------- Vec3 --- */
/* src/vec.zig:5-125 */
static inline ov3 V(double x, double y, double z) { ov3 r = {x, y, z}; return r; }
static inline ov3 vadd(ov3 a, ov3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline ov3 vsub(ov3 a, ov3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline ov3 vmul(ov3 a, ov3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline ov3 vscale(ov3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
static inline ov3 vdiv(ov3 a, double s) { return vscale(a, 1.0 / s); } /* vec.zig:37-39 */
static inline ov3 vneg(ov3 a) { return V(-a.x, -a.y, -a.z); }
static inline double vdot(ov3 a, ov3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline ov3 vcross(ov3 a, ov3 b) {
  return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double vlen2(ov3 a) { return vdot(a, a); }
static inline double vlen(ov3 a) { return sqrt(vlen2(a)); }
static inline ov3 vnorm(ov3 a) { return vdiv(a, vlen(a)); } /* vec.zig:66-70 */
static inline ov3 vlerp(ov3 a, ov3 b, double t) { return vadd(vscale(a, 1.0 - t), vscale(b, t)); }
static inline ov3 vmin(ov3 a, ov3 b) { return V(fmin(a.x, b.x), fmin(a.y, b.y), fmin(a.z, b.z)); }
static inline ov3 vmax(ov3 a, ov3 b) { return V(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)); }
static inline double vmaxc(ov3 a) { return fmax(a.x, fmax(a.y, a.z)); }
static inline double vget(ov3 a, int axis) { return axis == 0 ? a.x : (axis == 1 ? a.y : a.z); }
static inline int vnear_zero(ov3 a) { /* vec.zig:98-101 */
  const double eps = 1e-8;
  return fabs(a.x) < eps && fabs(a.y) < eps && fabs(a.z) < eps;
}
static inline int visfinite(ov3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
static inline ov3 vreflect(ov3 v, ov3 n) { return vsub(v, vscale(n, 2.0 * vdot(v, n))); }
static inline ov3 vrefract(ov3 uv, ov3 n, double eta) { /* vec.zig:119-124 */
  const double cos_theta = fmin(vdot(vneg(uv), n), 1.0);
  const ov3 r_perp = vscale(vadd(uv, vscale(n, cos_theta)), eta);
  const ov3 r_par = vscale(n, -sqrt(fabs(1.0 - vlen2(r_perp))));
  return vadd(r_perp, r_par);
}

/* ----------------------------------------------------------------- Rng --- */
/* src/rng.zig:10-88 (xoshiro256++ seeded through SplitMix64) */
typedef struct { uint64_t s[4]; } orng;

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t splitmix64(uint64_t* state) { /* rng.zig:82-88 */
  *state += 0x9E3779B97F4A7C15ULL;
  uint64_t z = *state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static inline orng rng_init(uint64_t seed) { /* rng.zig:13-18 */
  orng r;
  uint64_t sm = seed;
  for (int i = 0; i < 4; ++i) r.s[i] = splitmix64(&sm);
  return r;
}
static inline orng rng_for_stream(uint64_t seed, uint64_t stream) { /* rng.zig:22-25 */
  uint64_t sm = seed ^ (stream * 0x9E3779B97F4A7C15ULL);
  return rng_init(splitmix64(&sm));
}
static inline uint64_t rng_next(orng* r) { /* rng.zig:27-38 */
  uint64_t* s = r->s;
  const uint64_t result = rotl64(s[0] + s[3], 23) + s[0];
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl64(s[3], 45);
  return result;
}
static inline double rng_float(orng* r) { /* rng.zig:41-43 */
  return (double)(rng_next(r) >> 11) * 0x1.0p-53;
}
static inline double rng_range(orng* r, double lo, double hi) { /* rng.zig:46-48 */
  return lo + (hi - lo) * rng_float(r);
}
static inline uint64_t rng_below(orng* r, uint64_t n) { /* rng.zig:51-55 */
  return (uint64_t)(((unsigned __int128)rng_next(r) * n) >> 64);
}
static inline ov3 rng_unit_vector(orng* r) { /* rng.zig:58-63 */
  const double z = rng_range(r, -1.0, 1.0);
  const double phi = rng_range(r, 0.0, 2.0 * PI);
  const double rr = sqrt(fmax(0.0, 1.0 - z * z));
  double s, c;
  zt_sincos(phi, &s, &c);
  return V(rr * c, rr * s, z);
}
static inline ov3 rng_in_unit_sphere(orng* r) { /* rng.zig:66-71 */
  for (;;) {
    const double x = rng_range(r, -1, 1);
    const double y = rng_range(r, -1, 1);
    const double z = rng_range(r, -1, 1);
    const ov3 p = V(x, y, z);
    if (vlen2(p) < 1.0) return p;
  }
}
static inline ov3 rng_in_unit_disk(orng* r) { /* rng.zig:74-79 */
  for (;;) {
    const double x = rng_range(r, -1, 1);
    const double y = rng_range(r, -1, 1);
    const ov3 p = V(x, y, 0);
    if (vlen2(p) < 1.0) return p;
  }
}

/* ---------------------------------------------------------------- Aabb --- */
/* src/aabb.zig:7-88 */
typedef struct { ov3 min, max; } oaabb;
static inline oaabb aabb_empty(void) {
  oaabb a = {V(INFINITY, INFINITY, INFINITY), V(-INFINITY, -INFINITY, -INFINITY)};
  return a;
}
static inline oaabb aabb_from_points(ov3 a, ov3 b) { oaabb r = {vmin(a, b), vmax(a, b)}; return r; }
static inline oaabb aabb_merge(oaabb a, oaabb b) { oaabb r = {vmin(a.min, b.min), vmax(a.max, b.max)}; return r; }
static inline oaabb aabb_include(oaabb a, ov3 p) { oaabb r = {vmin(a.min, p), vmax(a.max, p)}; return r; }
static inline oaabb aabb_pad(oaabb a, double delta) { /* aabb.zig:30-39 */
  oaabb r = a;
  if (r.max.x - r.min.x < delta) { r.min.x -= delta / 2; r.max.x += delta / 2; }
  if (r.max.y - r.min.y < delta) { r.min.y -= delta / 2; r.max.y += delta / 2; }
  if (r.max.z - r.min.z < delta) { r.min.z -= delta / 2; r.max.z += delta / 2; }
  return r;
}
static inline int aabb_is_empty(oaabb a) { return a.min.x > a.max.x || a.min.y > a.max.y || a.min.z > a.max.z; }
static inline ov3 aabb_centroid(oaabb a) { return vscale(vadd(a.min, a.max), 0.5); }
static inline ov3 aabb_extent(oaabb a) { return vsub(a.max, a.min); }
static inline double aabb_sa(oaabb a) { /* aabb.zig:53-57 */
  if (aabb_is_empty(a)) return 0;
  const ov3 e = aabb_extent(a);
  return 2.0 * (e.x * e.y + e.y * e.z + e.z * e.x);
}
static inline int aabb_longest_axis(oaabb a) { /* aabb.zig:59-63 */
  const ov3 e = aabb_extent(a);
  if (e.x >= e.y && e.x >= e.z) return 0;
  return e.y >= e.z ? 1 : 2;
}
/* Slab test, aabb.zig:68-83. NaN (0*inf) compares false and leaves the
 * interval unchanged. */
static inline int aabb_hit(const ov3* bmin, const ov3* bmax, ov3 o, ov3 inv, double tmin, double tmax,
                           double* tout) {
  double lo = tmin, hi = tmax;
  for (int axis = 0; axis < 3; ++axis) {
    const double iv = vget(inv, axis);
    const double oo = vget(o, axis);
    double t0 = (vget(*bmin, axis) - oo) * iv;
    double t1 = (vget(*bmax, axis) - oo) * iv;
    if (iv < 0) { const double tmp = t0; t0 = t1; t1 = tmp; }
    if (t0 > lo) lo = t0;
    if (t1 < hi) hi = t1;
    if (hi < lo) return 0;
  }
  *tout = lo;
  return 1;
}
static inline ov3 vinverse(ov3 d) { return V(1.0 / d.x, 1.0 / d.y, 1.0 / d.z); } /* aabb.zig:86-88 */

/* ------------------------------------------------------------ Geometry --- */
/* src/geometry.zig */
static inline ov3 P3(const double* p) { return V(p[0], p[1], p[2]); }
static inline ov3 ray_at(ov3 o, ov3 d, double t) { return vadd(o, vscale(d, t)); } /* ray.zig:12-14 */

static inline void hit_make(ov3 o, ov3 d, double t, ov3 outward, uint32_t mat, ohit* h) { /* geometry.zig:19-29 */
  const int front = vdot(d, outward) < 0;
  h->t = t;
  h->point = ray_at(o, d, t);
  h->normal = front ? outward : vneg(outward);
  h->front_face = (uint32_t)front;
  h->material = mat;
}

static int sphere_intersect(const oshape* s, ov3 o, ov3 d, double tmin, double tmax, ohit* h) {
  /* geometry.zig:37-52 */
  const ov3 center = P3(s->p);
  const double radius = s->p[3];
  const ov3 oc = vsub(center, o);
  const double a = vlen2(d);
  const double hh = vdot(d, oc);
  const double c = vlen2(oc) - radius * radius;
  const double disc = hh * hh - a * c;
  if (disc < 0) return 0;
  const double sq = sqrt(disc);
  double t = (hh - sq) / a;
  if (t <= tmin || t >= tmax) {
    t = (hh + sq) / a;
    if (t <= tmin || t >= tmax) return 0;
  }
  const ov3 outward = vdiv(vsub(ray_at(o, d, t), center), radius);
  hit_make(o, d, t, outward, s->material, h);
  return 1;
}

static int plane_intersect(const oshape* s, ov3 o, ov3 d, double tmin, double tmax, ohit* h) {
  /* geometry.zig:67-73 */
  const ov3 point = P3(s->p), normal = P3(s->p + 3);
  const double denom = vdot(normal, d);
  if (fabs(denom) < 1e-12) return 0;
  const double t = vdot(vsub(point, o), normal) / denom;
  if (t <= tmin || t >= tmax) return 0;
  hit_make(o, d, t, normal, s->material, h);
  return 1;
}

static int triangle_intersect(const oshape* s, ov3 o, ov3 d, double tmin, double tmax, ohit* h) {
  /* Moller-Trumbore, geometry.zig:83-99 */
  const ov3 v0 = P3(s->p), v1 = P3(s->p + 3), v2 = P3(s->p + 6);
  const ov3 e1 = vsub(v1, v0);
  const ov3 e2 = vsub(v2, v0);
  const ov3 p = vcross(d, e2);
  const double det = vdot(e1, p);
  if (fabs(det) < 1e-12) return 0;
  const double inv_det = 1.0 / det;
  const ov3 sv = vsub(o, v0);
  const double u = vdot(sv, p) * inv_det;
  if (u < 0 || u > 1) return 0;
  const ov3 q = vcross(sv, e1);
  const double v = vdot(d, q) * inv_det;
  if (v < 0 || u + v > 1) return 0;
  const double t = vdot(e2, q) * inv_det;
  if (t <= tmin || t >= tmax) return 0;
  hit_make(o, d, t, vnorm(vcross(e1, e2)), s->material, h);
  return 1;
}

static inline int shape_intersect(const oshape* s, ov3 o, ov3 d, double tmin, double tmax, ohit* h,
                                  ostats* st) { /* geometry.zig:106-125 */
  switch (s->kind) {
    case O_SPHERE: if (st) st->sphere_tests++; return sphere_intersect(s, o, d, tmin, tmax, h);
    case O_TRIANGLE: if (st) st->tri_tests++; return triangle_intersect(s, o, d, tmin, tmax, h);
    default: if (st) st->plane_tests++; return plane_intersect(s, o, d, tmin, tmax, h);
  }
}

static inline int shape_bounds(const oshape* s, oaabb* b) { /* geometry.zig:241-247 */
  if (s->kind == O_SPHERE) { /* geometry.zig:54-57 */
    const double ar = fabs(s->p[3]);
    const ov3 r = V(ar, ar, ar), c = P3(s->p);
    b->min = vsub(c, r);
    b->max = vadd(c, r);
    return 1;
  }
  if (s->kind == O_TRIANGLE) { /* geometry.zig:101-103 */
    *b = aabb_pad(aabb_include(aabb_from_points(P3(s->p), P3(s->p + 3)), P3(s->p + 6)), 1e-6);
    return 1;
  }
  return 0;
}

/* intersectAll, geometry.zig:129-139; prim ids are base + index. */
static int intersect_all(const oshape* shapes, size_t n, int32_t base, ov3 o, ov3 d, double tmin,
                         double tmax, ohit* best, ostats* st) {
  double closest = tmax;
  int found = 0;
  ohit h;
  for (size_t i = 0; i < n; ++i) {
    if (shape_intersect(&shapes[i], o, d, tmin, closest, &h, st)) {
      closest = h.t;
      *best = h;
      best->prim = base + (int32_t)i;
      found = 1;
    }
  }
  return found;
}

/* ----------------------------------------------------------- Material --- */
/* src/material.zig */
static inline ov3 material_emitted(const omaterial* m, const ohit* h) { /* material.zig:26-32 */
  if (m->kind == O_EMISSIVE && h->front_face) return m->color;
  return V(0, 0, 0);
}

static inline double schlick(double cosine, double eta) { /* material.zig:66-70 */
  double r0 = (1.0 - eta) / (1.0 + eta);
  r0 *= r0;
  return r0 + (1.0 - r0) * zt_pow5(1.0 - cosine);
}

/* material.zig:34-62; returns 1 with attenuation and scattered ray. */
static int material_scatter(const omaterial* m, ov3 in_dir, const ohit* h, orng* rng, ov3* atten,
                            ov3* out_o, ov3* out_d) {
  switch (m->kind) {
    case O_LAMBERTIAN: {
      ov3 dir = vadd(h->normal, rng_unit_vector(rng));
      if (vnear_zero(dir)) dir = h->normal;
      *atten = m->color;
      *out_o = h->point;
      *out_d = vnorm(dir);
      return 1;
    }
    case O_METAL: {
      ov3 dir = vreflect(vnorm(in_dir), h->normal);
      if (m->param > 0) dir = vnorm(vadd(dir, vscale(rng_unit_vector(rng), m->param)));
      if (vdot(dir, h->normal) <= 0) return 0;
      *atten = m->color;
      *out_o = h->point;
      *out_d = dir;
      return 1;
    }
    case O_DIELECTRIC: {
      const double eta = h->front_face ? 1.0 / m->param : m->param;
      const ov3 unit = vnorm(in_dir);
      const double cos_theta = fmin(vdot(vneg(unit), h->normal), 1.0);
      const double sin_theta = sqrt(fmax(0.0, 1.0 - cos_theta * cos_theta));
      const int cannot_refract = eta * sin_theta > 1.0;
      ov3 dir;
      /* material.zig:54: `or` short-circuits, so no draw under TIR. */
      if (cannot_refract || schlick(cos_theta, eta) > rng_float(rng))
        dir = vreflect(unit, h->normal);
      else
        dir = vrefract(unit, h->normal, eta);
      *atten = V(1, 1, 1);
      *out_o = h->point;
      *out_d = dir;
      return 1;
    }
    default:
      return 0;
  }
}

/* ------------------------------------------------------------- Camera --- */
/* src/camera.zig:29-67 */
static void camera_init(const ocamera_config* cfg, double aspect, ocamera* c) {
  const double theta = cfg->vfov * (PI / 180.0); /* std.math.degreesToRadians */
  const double half_h = tan(theta / 2);
  const double viewport_h = 2.0 * half_h;
  const double viewport_w = aspect * viewport_h;
  const ov3 w = vnorm(vsub(cfg->look_from, cfg->look_at));
  const ov3 u = vnorm(vcross(cfg->up, w));
  const ov3 v = vcross(w, u);
  const double focus = cfg->has_focus_dist ? cfg->focus_dist : vlen(vsub(cfg->look_from, cfg->look_at));
  const ov3 horizontal = vscale(u, viewport_w * focus);
  const ov3 vertical = vscale(v, -viewport_h * focus);
  const ov3 upper_left =
      vsub(vsub(vsub(cfg->look_from, vscale(w, focus)), vscale(horizontal, 0.5)), vscale(vertical, 0.5));
  c->origin = cfg->look_from;
  c->upper_left = upper_left;
  c->horizontal = horizontal;
  c->vertical = vertical;
  c->u = u;
  c->v = v;
  c->lens_radius = cfg->aperture / 2;
}

static inline void camera_ray(const ocamera* c, double s, double t, orng* rng, ov3* ro, ov3* rd) {
  ov3 origin = c->origin;
  if (c->lens_radius > 0) {
    const ov3 d = vscale(rng_in_unit_disk(rng), c->lens_radius);
    origin = vadd(vadd(origin, vscale(c->u, d.x)), vscale(c->v, d.y));
  }
  const ov3 target = vadd(vadd(c->upper_left, vscale(c->horizontal, s)), vscale(c->vertical, t));
  *ro = origin;
  *rd = vnorm(vsub(target, origin));
}

static inline ov3 background_radiance(const obackground* bg, ov3 dir) { /* scene.zig:20-28 */
  if (bg->kind == O_BG_SOLID) return bg->a;
  const double t = fmax(0.0, fmin(vnorm(dir).y, 1.0)); /* std.math.clamp */
  return vlerp(bg->a, bg->b, t);
}

/* ---------------------------------------------------------------- Scene --- */
struct oscene {
  omaterial* mats;
  size_t n_mats;
  oshape* shapes; /* bounded, in insertion order */
  size_t n_shapes;
  oshape* planes; /* unbounded, in insertion order */
  size_t n_planes;
  ocamera_config camera;
  obackground background;
  int built;
  onode* nodes;
  size_t n_nodes;
  uint32_t* indices;
  olight* lights;
  double* cdf;
  size_t n_lights;
  double total;
};

/* ------------------------------------------------------------------ BVH --- */
/* src/bvh.zig:16-263 */
#define BIN_COUNT 12
#define MAX_LEAF_SIZE 4
#define BVH_MAX_DEPTH 64
#define TRAVERSAL_COST 1.0

typedef struct {
  onode* nodes;
  size_t n_nodes;
  uint32_t* indices;
  const oaabb* boxes;
  const ov3* centroids;
} obuilder;

static inline size_t bin_of(double c, double lo, double extent) { /* bvh.zig:258-262 */
  const double f = (c - lo) / extent * (double)BIN_COUNT;
  const double cl = fmax(0.0, fmin(f, (double)(BIN_COUNT - 1)));
  return (size_t)cl;
}

typedef struct { int axis; size_t bin; double cost; int valid; } osplit;

static osplit find_split(obuilder* b, const uint32_t* range, size_t count, oaabb bounds, oaabb cb) {
  /* bvh.zig:211-256 */
  osplit best = {0, 0, 0, 0};
  const double parent_area = aabb_sa(bounds);
  if (parent_area <= 0) return best;
  for (int axis = 0; axis < 3; ++axis) {
    const double lo = vget(cb.min, axis);
    const double extent = vget(cb.max, axis) - lo;
    if (!(extent > 0)) continue;
    oaabb bin_bounds[BIN_COUNT];
    size_t bin_counts[BIN_COUNT];
    for (int i = 0; i < BIN_COUNT; ++i) { bin_bounds[i] = aabb_empty(); bin_counts[i] = 0; }
    for (size_t j = 0; j < count; ++j) {
      const uint32_t idx = range[j];
      const size_t bb = bin_of(vget(b->centroids[idx], axis), lo, extent);
      bin_counts[bb] += 1;
      bin_bounds[bb] = aabb_merge(bin_bounds[bb], b->boxes[idx]);
    }
    double right_area[BIN_COUNT];
    size_t right_count[BIN_COUNT];
    oaabb acc = aabb_empty();
    size_t acc_n = 0;
    for (int i = BIN_COUNT - 1; i >= 0; --i) {
      acc = aabb_merge(acc, bin_bounds[i]);
      acc_n += bin_counts[i];
      right_area[i] = aabb_sa(acc);
      right_count[i] = acc_n;
    }
    acc = aabb_empty();
    acc_n = 0;
    for (int bb = 0; bb < BIN_COUNT - 1; ++bb) {
      acc = aabb_merge(acc, bin_bounds[bb]);
      acc_n += bin_counts[bb];
      const size_t rn = right_count[bb + 1];
      if (acc_n == 0 || rn == 0) continue;
      const double cost =
          TRAVERSAL_COST + (aabb_sa(acc) * (double)acc_n + right_area[bb + 1] * (double)rn) / parent_area;
      if (!best.valid || cost < best.cost) {
        best.axis = axis;
        best.bin = (size_t)bb;
        best.cost = cost;
        best.valid = 1;
      }
    }
  }
  return best;
}

static void subdivide(obuilder* b, size_t node_idx, size_t level);

static void make_children(obuilder* b, size_t node_idx, uint32_t first, uint32_t left_count, uint32_t count,
                          size_t level) { /* bvh.zig:187-195 */
  const uint32_t left = (uint32_t)b->n_nodes;
  onode* nl = &b->nodes[b->n_nodes++];
  nl->bmin = aabb_empty().min; nl->bmax = aabb_empty().max; nl->first = first; nl->count = left_count;
  onode* nr = &b->nodes[b->n_nodes++];
  nr->bmin = aabb_empty().min; nr->bmax = aabb_empty().max; nr->first = first + left_count; nr->count = count - left_count;
  b->nodes[node_idx].first = left;
  b->nodes[node_idx].count = 0;
  subdivide(b, left, level + 1);
  subdivide(b, left + 1, level + 1);
}

/* Stable merge sort of indices by centroid[axis] (std.mem.sort is stable). */
static void stable_sort_axis(uint32_t* a, size_t n, const ov3* centroids, int axis, uint32_t* tmp) {
  if (n < 2) return;
  const size_t h = n / 2;
  stable_sort_axis(a, h, centroids, axis, tmp);
  stable_sort_axis(a + h, n - h, centroids, axis, tmp);
  size_t i = 0, j = h, k = 0;
  while (i < h && j < n) {
    /* take from the right only when strictly less: keeps equal keys in order */
    if (vget(centroids[a[j]], axis) < vget(centroids[a[i]], axis)) tmp[k++] = a[j++];
    else tmp[k++] = a[i++];
  }
  while (i < h) tmp[k++] = a[i++];
  while (j < n) tmp[k++] = a[j++];
  memcpy(a, tmp, n * sizeof(uint32_t));
}

static void split_median(obuilder* b, size_t node_idx, uint32_t* range, size_t count, oaabb cb, size_t level) {
  /* bvh.zig:197-209 */
  const int axis = aabb_longest_axis(cb);
  uint32_t* tmp = (uint32_t*)malloc(count * sizeof(uint32_t));
  stable_sort_axis(range, count, b->centroids, axis, tmp);
  free(tmp);
  const onode node = b->nodes[node_idx];
  make_children(b, node_idx, node.first, node.count / 2, node.count, level);
}

static void subdivide(obuilder* b, size_t node_idx, size_t level) { /* bvh.zig:148-185 */
  onode* node = &b->nodes[node_idx];
  const uint32_t first = node->first;
  const uint32_t count = node->count;
  uint32_t* range = b->indices + first;
  oaabb bounds = aabb_empty(), cb = aabb_empty();
  for (uint32_t j = 0; j < count; ++j) {
    const uint32_t i = range[j];
    bounds = aabb_merge(bounds, b->boxes[i]);
    cb = aabb_include(cb, b->centroids[i]);
  }
  node->bmin = bounds.min;
  node->bmax = bounds.max;
  if (count <= 1 || level >= BVH_MAX_DEPTH) return;
  const double leaf_cost = (double)count;
  const osplit split = find_split(b, range, count, bounds, cb);
  if (!split.valid) {
    if (count <= MAX_LEAF_SIZE) return;
    split_median(b, node_idx, range, count, cb, level);
    return;
  }
  if (count <= MAX_LEAF_SIZE && split.cost >= leaf_cost) return;
  const int axis = split.axis;
  const double lo = vget(cb.min, axis);
  const double extent = vget(cb.max, axis) - lo;
  uint32_t mid = 0;
  for (uint32_t j = 0; j < count; ++j) {
    const uint32_t idx = range[j];
    if (bin_of(vget(b->centroids[idx], axis), lo, extent) <= split.bin) {
      const uint32_t tmp = range[mid];
      range[mid] = range[j];
      range[j] = tmp;
      mid += 1;
    }
  }
  make_children(b, node_idx, first, mid, count, level);
}

static int bvh_build(oscene* s) { /* bvh.zig:41-67 */
  const size_t n = s->n_shapes;
  s->nodes = NULL;
  s->n_nodes = 0;
  s->indices = NULL;
  if (n == 0) return 0;
  if (n > 0xFFFFFFFFu / 2) return -3;
  s->indices = (uint32_t*)malloc(n * sizeof(uint32_t));
  oaabb* boxes = (oaabb*)malloc(n * sizeof(oaabb));
  ov3* centroids = (ov3*)malloc(n * sizeof(ov3));
  s->nodes = (onode*)malloc((2 * n - 1) * sizeof(onode));
  if (!s->indices || !boxes || !centroids || !s->nodes) { free(boxes); free(centroids); return -2; }
  for (size_t i = 0; i < n; ++i) {
    s->indices[i] = (uint32_t)i;
    shape_bounds(&s->shapes[i], &boxes[i]);
    centroids[i] = aabb_centroid(boxes[i]);
  }
  obuilder b = {s->nodes, 0, s->indices, boxes, centroids};
  onode* root = &b.nodes[b.n_nodes++];
  root->bmin = aabb_empty().min;
  root->bmax = aabb_empty().max;
  root->first = 0;
  root->count = (uint32_t)n;
  subdivide(&b, 0, 0);
  s->n_nodes = b.n_nodes;
  free(boxes);
  free(centroids);
  return 0;
}

/* Bvh.intersect, bvh.zig:80-126. */
static int bvh_intersect(const oscene* s, ov3 o, ov3 d, double tmin, double tmax, ohit* best, ostats* st) {
  if (s->n_nodes == 0) return 0;
  const ov3 inv = vinverse(d);
  double closest = tmax;
  int found = 0;
  struct { uint32_t node; double t; } stack[BVH_MAX_DEPTH + 2];
  size_t sp = 0;
  double t;
  if (st) st->slab_tests++;
  if (aabb_hit(&s->nodes[0].bmin, &s->nodes[0].bmax, o, inv, tmin, closest, &t)) {
    stack[0].node = 0;
    stack[0].t = t;
    sp = 1;
  }
  ohit h;
  while (sp > 0) {
    sp -= 1;
    const uint32_t ni = stack[sp].node;
    const double et = stack[sp].t;
    if (et > closest) continue;
    if (st) st->node_pops++;
    const onode* node = &s->nodes[ni];
    if (node->count > 0) {
      for (uint32_t k = 0; k < node->count; ++k) {
        const uint32_t idx = s->indices[node->first + k];
        if (shape_intersect(&s->shapes[idx], o, d, tmin, closest, &h, st)) {
          closest = h.t;
          *best = h;
          best->prim = (int32_t)idx;
          found = 1;
        }
      }
      continue;
    }
    const uint32_t l = node->first;
    double tl, tr;
    if (st) st->slab_tests += 2;
    const int hl = aabb_hit(&s->nodes[l].bmin, &s->nodes[l].bmax, o, inv, tmin, closest, &tl);
    const int hr = aabb_hit(&s->nodes[l + 1].bmin, &s->nodes[l + 1].bmax, o, inv, tmin, closest, &tr);
    if (hl && hr) {
      const int near_left = tl <= tr;
      if (near_left) {
        stack[sp].node = l + 1; stack[sp].t = tr;
        stack[sp + 1].node = l; stack[sp + 1].t = tl;
      } else {
        stack[sp].node = l; stack[sp].t = tl;
        stack[sp + 1].node = l + 1; stack[sp + 1].t = tr;
      }
      sp += 2;
    } else if (hl) {
      stack[sp].node = l; stack[sp].t = tl;
      sp += 1;
    } else if (hr) {
      stack[sp].node = l + 1; stack[sp].t = tr;
      sp += 1;
    }
  }
  return found;
}

/* Scene.intersect, scene.zig:108-116. */
static int scene_intersect(const oscene* s, ov3 o, ov3 d, double tmin, double tmax, ohit* out, ostats* st) {
  ohit best;
  int found;
  if (s->built)
    found = bvh_intersect(s, o, d, tmin, tmax, &best, st);
  else
    found = intersect_all(s->shapes, s->n_shapes, 0, o, d, tmin, tmax, &best, st);
  const double limit = found ? best.t : tmax;
  ohit hp;
  if (intersect_all(s->planes, s->n_planes, (int32_t)s->n_shapes, o, d, tmin, limit, &hp, st)) {
    best = hp;
    found = 1;
  }
  if (found) *out = best;
  return found;
}

/* --------------------------------------------------------------- Lights --- */
/* src/light.zig */
static inline double luminance(ov3 c) { return 0.2126 * c.x + 0.7152 * c.y + 0.0722 * c.z; }
static inline double triangle_area(const oshape* t) { /* light.zig:42-44 */
  const ov3 v0 = P3(t->p), v1 = P3(t->p + 3), v2 = P3(t->p + 6);
  return 0.5 * vlen(vcross(vsub(v1, v0), vsub(v2, v0)));
}
static inline int sphere_outside(const oshape* s, ov3 origin) { /* light.zig:47-50 */
  const double d = vlen(vsub(P3(s->p), origin));
  return d > fabs(s->p[3]) * (1 + 1e-9);
}
static inline void onb_basis(ov3 w, ov3* u, ov3* v) { /* light.zig:53-57 */
  const ov3 a = fabs(w.x) > 0.9 ? V(0, 1, 0) : V(1, 0, 0);
  *v = vnorm(vcross(w, a));
  *u = vcross(*v, w);
}

static int lights_build(oscene* s) { /* light.zig:68-94 */
  s->lights = (olight*)malloc((s->n_shapes ? s->n_shapes : 1) * sizeof(olight));
  if (!s->lights) return -2;
  size_t n = 0;
  for (size_t i = 0; i < s->n_shapes; ++i) {
    const oshape* sh = &s->shapes[i];
    double area;
    if (sh->kind == O_TRIANGLE) area = triangle_area(sh);
    else if (sh->kind == O_SPHERE) area = sh->p[3] > 0 ? 4 * PI * sh->p[3] * sh->p[3] : 0;
    else continue;
    const omaterial* m = &s->mats[sh->material];
    if (m->kind != O_EMISSIVE) continue;
    const double weight = luminance(m->color) * area;
    if (!(weight > 0) || !isfinite(weight)) continue;
    s->lights[n].shape = *sh;
    s->lights[n].radiance = m->color;
    s->lights[n].weight = weight;
    n++;
  }
  s->n_lights = n;
  s->cdf = (double*)malloc((n ? n : 1) * sizeof(double));
  if (!s->cdf) return -2;
  double sum = 0;
  for (size_t i = 0; i < n; ++i) {
    sum += s->lights[i].weight;
    s->cdf[i] = sum;
  }
  s->total = sum;
  return 0;
}

static inline const olight* lights_pick(const oscene* s, orng* rng) { /* light.zig:106-115 */
  const double x = rng_float(rng) * s->total;
  size_t lo = 0, hi = s->n_lights - 1;
  while (lo < hi) {
    const size_t mid = (lo + hi) / 2;
    if (s->cdf[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  return &s->lights[lo];
}

/* Lights.sample, light.zig:120-166. */
static int lights_sample(const oscene* s, ov3 origin, orng* rng, ov3* odir, double* odist, ov3* orad,
                         double* opdf) {
  if (s->n_lights == 0) return 0;
  const olight* light = lights_pick(s, rng);
  const double select = light->weight / s->total;
  if (light->shape.kind == O_TRIANGLE) {
    const oshape* t = &light->shape;
    const ov3 v0 = P3(t->p), v1 = P3(t->p + 3), v2 = P3(t->p + 6);
    const double su = sqrt(rng_float(rng));
    const double b2 = rng_float(rng);
    const ov3 p = vadd(vadd(vscale(v0, 1 - su), vscale(v1, su * (1 - b2))), vscale(v2, su * b2));
    const ov3 to = vsub(p, origin);
    const double dist = vlen(to);
    if (dist < 1e-9) return 0;
    const ov3 dir = vscale(to, 1 / dist);
    const ov3 n = vnorm(vcross(vsub(v1, v0), vsub(v2, v0)));
    const double cos_l = -vdot(dir, n);
    if (cos_l <= 1e-9) return 0;
    *odir = dir;
    *odist = dist;
    *orad = light->radiance;
    *opdf = select * dist * dist / (cos_l * triangle_area(t));
    return 1;
  }
  /* sphere, light.zig:143-163 */
  const oshape* sp = &light->shape;
  if (!sphere_outside(sp, origin)) return 0;
  const ov3 center = P3(sp->p);
  const double radius = sp->p[3];
  const ov3 axis = vsub(center, origin);
  const double d2 = vlen2(axis);
  const ov3 w = vscale(axis, 1 / sqrt(d2));
  const double cos_max = sqrt(fmax(0.0, 1 - radius * radius / d2));
  const double cos_t = 1 - rng_float(rng) * (1 - cos_max);
  const double sin_t = sqrt(fmax(0.0, 1 - cos_t * cos_t));
  const double phi = 2 * PI * rng_float(rng);
  ov3 bu, bv;
  onb_basis(w, &bu, &bv);
  double sphi, cphi;
  zt_sincos(phi, &sphi, &cphi);
  const ov3 dir = vnorm(vadd(vadd(vscale(bu, sin_t * cphi), vscale(bv, sin_t * sphi)), vscale(w, cos_t)));
  ohit h;
  if (!sphere_intersect(sp, origin, dir, 0, INFINITY, &h)) return 0;
  if (!h.front_face) return 0;
  *odir = dir;
  *odist = h.t;
  *orad = light->radiance;
  *opdf = select / (2 * PI * (1 - cos_max));
  return 1;
}

/* Lights.pdfHit, light.zig:171-198. */
static double lights_pdf_hit(const oscene* s, ov3 origin, const ohit* hit, ostats* st) {
  if (st) st->pdfhit_calls++;
  const ov3 to = vsub(hit->point, origin);
  const double dist = vlen(to);
  if (dist < 1e-9) return 0;
  const ov3 dir = vscale(to, 1 / dist);
  double pdf = 0;
  ohit h;
  for (size_t i = 0; i < s->n_lights; ++i) {
    const olight* light = &s->lights[i];
    const double select = light->weight / s->total;
    if (st) st->pdfhit_light_tests++;
    if (light->shape.kind == O_TRIANGLE) {
      if (!triangle_intersect(&light->shape, origin, dir, 1e-9, INFINITY, &h)) continue;
      if (fabs(h.t - dist) > 1e-6 * dist || !h.front_face) continue;
      pdf += select * dist * dist / (-vdot(dir, h.normal) * triangle_area(&light->shape));
    } else if (light->shape.kind == O_SPHERE) {
      if (!sphere_outside(&light->shape, origin)) continue;
      if (!sphere_intersect(&light->shape, origin, dir, 1e-9, INFINITY, &h)) continue;
      if (fabs(h.t - dist) > 1e-6 * dist || !h.front_face) continue;
      const double r = light->shape.p[3];
      const double d2 = vlen2(vsub(P3(light->shape.p), origin));
      const double cos_max = sqrt(fmax(0.0, 1 - r * r / d2));
      pdf += select / (2 * PI * (1 - cos_max));
    }
  }
  return pdf;
}

/* ------------------------------------------------------------ Integrator --- */
/* src/render.zig */
#define RAY_EPSILON 1e-4
#define ROULETTE_DEPTH 4

static inline double power_weight(double a, double b) { /* render.zig:38-41 */
  const double a2 = a * a;
  return a2 / (a2 + b * b);
}

static ov3 direct_light(const oscene* s, ov3 albedo, const ohit* hit, orng* rng, ostats* st) {
  /* render.zig:46-56 */
  ov3 ldir, lrad;
  double ldist, lpdf;
  if (st) st->nee_samples++;
  if (!lights_sample(s, hit->point, rng, &ldir, &ldist, &lrad, &lpdf)) return V(0, 0, 0);
  const double cos_s = vdot(hit->normal, ldir);
  if (cos_s <= 0 || !(lpdf > 0)) return V(0, 0, 0);
  ohit sh;
  if (st) st->shadow_rays++;
  if (scene_intersect(s, hit->point, ldir, RAY_EPSILON, ldist * (1 - 1e-6), &sh, st)) return V(0, 0, 0);
  const double bsdf_pdf = cos_s / PI;
  const double scale = cos_s / (PI * lpdf) * power_weight(lpdf, bsdf_pdf);
  return vscale(vmul(albedo, lrad), scale);
}

/* traceWith, render.zig:61-102.  first_prim/path_len are instrumentation. */
static ov3 trace_with(const oscene* s, ov3 ro, ov3 rd, orng* rng, uint64_t max_depth, int light_sampling,
                      ostats* st, int32_t* first_prim, uint32_t* path_len) {
  const int use_nee = light_sampling && s->n_lights > 0;
  ov3 radiance = V(0, 0, 0), throughput = V(1, 1, 1);
  ov3 prev_origin = V(0, 0, 0);
  double prev_pdf = 0;
  uint32_t n_ext = 0;
  if (first_prim) *first_prim = -1;
  for (uint64_t depth = 0; depth < max_depth; ++depth) {
    ohit hit;
    n_ext++;
    if (st) st->ext_rays++;
    if (!scene_intersect(s, ro, rd, RAY_EPSILON, INFINITY, &hit, st)) {
      if (path_len) *path_len = n_ext;
      return vadd(radiance, vmul(throughput, background_radiance(&s->background, rd)));
    }
    if (st) st->hits++;
    if (depth == 0 && first_prim) *first_prim = hit.prim;
    const omaterial* mat = &s->mats[hit.material];
    const ov3 le = material_emitted(mat, &hit);
    if (vmaxc(le) > 0) {
      const double w = prev_pdf > 0 ? power_weight(prev_pdf, lights_pdf_hit(s, prev_origin, &hit, st)) : 1.0;
      radiance = vadd(radiance, vscale(vmul(throughput, le), w));
    }
    if (mat->kind == O_LAMBERTIAN && use_nee)
      radiance = vadd(radiance, vmul(throughput, direct_light(s, mat->color, &hit, rng, st)));
    ov3 atten, so, sd;
    if (!material_scatter(mat, rd, &hit, rng, &atten, &so, &sd)) break;
    throughput = vmul(throughput, atten);
    prev_pdf = (use_nee && mat->kind == O_LAMBERTIAN) ? fmax(vdot(sd, hit.normal), 0) / PI : 0;
    prev_origin = hit.point;
    ro = so;
    rd = sd;
    if (depth + 1 >= ROULETTE_DEPTH) {
      const double p = fmin(vmaxc(throughput), 0.95);
      if (p <= 0 || rng_float(rng) >= p) break;
      throughput = vdiv(throughput, p);
    }
  }
  if (path_len) *path_len = n_ext;
  return radiance;
}

static int options_valid(const ooptions* o);

/* traceWith with detached sampling for the differentiable form: the scene's
 * materials drive roulette (throughput tp0), the light pick and the MIS
 * weights; `theta` (3 per material) drives the contributions.  With theta =
 * the scene's colours this is trace_with operation for operation. */
static ov3 trace_params(const oscene* s, const double* theta, ov3 ro, ov3 rd, orng* rng, uint64_t max_depth,
                        int light_sampling) {
  const int use_nee = light_sampling && s->n_lights > 0;
  ov3 radiance = V(0, 0, 0), tp = V(1, 1, 1), tp0 = V(1, 1, 1), prev_origin = V(0, 0, 0);
  double prev_pdf = 0;
  for (uint64_t depth = 0; depth < max_depth; ++depth) {
    ohit hit;
    if (!scene_intersect(s, ro, rd, RAY_EPSILON, INFINITY, &hit, NULL))
      return vadd(radiance, vmul(tp, background_radiance(&s->background, rd)));
    const uint32_t m = hit.material;
    const omaterial* mat = &s->mats[m];
    const ov3 th = P3(theta + 3 * (size_t)m);
    const ov3 le0 = material_emitted(mat, &hit);
    if (vmaxc(le0) > 0) {
      const double w = prev_pdf > 0 ? power_weight(prev_pdf, lights_pdf_hit(s, prev_origin, &hit, NULL)) : 1.0;
      radiance = vadd(radiance, vscale(vmul(tp, th), w));
    }
    if (mat->kind == O_LAMBERTIAN && use_nee) {
      ov3 direct = V(0, 0, 0), ldir, lrad0;
      double ldist, lpdf;
      orng probe = *rng;
      /* which light the pick chooses: light.zig:106-115 on a copy of the stream */
      const olight* picked = s->n_lights ? lights_pick(s, &probe) : NULL;
      if (lights_sample(s, hit.point, rng, &ldir, &ldist, &lrad0, &lpdf)) {
        const double cos_s = vdot(hit.normal, ldir);
        ohit sh;
        if (!(cos_s <= 0 || !(lpdf > 0)) &&
            !scene_intersect(s, hit.point, ldir, RAY_EPSILON, ldist * (1 - 1e-6), &sh, NULL)) {
          const double bsdf_pdf = cos_s / PI;
          const double scale = cos_s / (PI * lpdf) * power_weight(lpdf, bsdf_pdf);
          direct = vscale(vmul(th, P3(theta + 3 * (size_t)picked->shape.material)), scale);
        }
      }
      radiance = vadd(radiance, vmul(tp, direct));
    }
    ov3 atten0, so, sd;
    if (!material_scatter(mat, rd, &hit, rng, &atten0, &so, &sd)) break;
    const ov3 atten = (mat->kind == O_LAMBERTIAN || mat->kind == O_METAL) ? th : atten0;
    tp = vmul(tp, atten);
    tp0 = vmul(tp0, atten0);
    prev_pdf = (use_nee && mat->kind == O_LAMBERTIAN) ? fmax(vdot(sd, hit.normal), 0) / PI : 0;
    prev_origin = hit.point;
    ro = so;
    rd = sd;
    if (depth + 1 >= ROULETTE_DEPTH) {
      const double p = fmin(vmaxc(tp0), 0.95);
      if (p <= 0 || rng_float(rng) >= p) break;
      tp = vdiv(tp, p);
      tp0 = vdiv(tp0, p);
    }
  }
  return radiance;
}

int ozt_render_params(const oscene* s, const ooptions* o, const double* theta, double* out) {
  if (!options_valid(o)) return -1;
  ocamera cam;
  camera_init(&s->camera, (double)o->width / (double)o->height, &cam);
  const double w = (double)o->width, h = (double)o->height, inv_spp = 1.0 / (double)o->spp;
  for (uint64_t y = 0; y < o->height; ++y)
    for (uint64_t x = 0; x < o->width; ++x) {
      orng rng = rng_for_stream(o->seed, y * o->width + x);
      ov3 sum = V(0, 0, 0);
      for (uint64_t i = 0; i < o->spp; ++i) {
        const double sx = ((double)x + rng_float(&rng)) / w;
        const double ty = ((double)y + rng_float(&rng)) / h;
        ov3 ro, rd;
        camera_ray(&cam, sx, ty, &rng, &ro, &rd);
        const ov3 c = trace_params(s, theta, ro, rd, &rng, o->max_depth, (int)o->light_sampling);
        if (visfinite(c)) sum = vadd(sum, c);
      }
      const ov3 px = vscale(sum, inv_spp);
      double* dst = out + 3 * (y * o->width + x);
      dst[0] = px.x;
      dst[1] = px.y;
      dst[2] = px.z;
    }
  return 0;
}

/* ---------------------------------------------------------------- Render --- */
/* render.zig:104-180 */
typedef struct {
  const oscene* s;
  ocamera cam;
  const ooptions* o;
  double* out;
  uint64_t tiles_x, tile_count;
  atomic_ulong next_tile;
  pthread_mutex_t stats_lock;
  ostats* stats;
  /* pixel-subset mode */
  const uint64_t* pixels;
  size_t n_pixels;
  /* optional: per pixel, the mean of the squared luminance of its samples */
  double* moments;
} octx;

static void render_pixel(octx* c, uint64_t x, uint64_t y, double* dst, ostats* st) { /* render.zig:133-144 */
  const double w = (double)c->o->width, h = (double)c->o->height;
  const double inv_spp = 1.0 / (double)c->o->spp;
  orng rng = rng_for_stream(c->o->seed, y * c->o->width + x);
  ov3 sum = V(0, 0, 0);
  double lum2 = 0;
  for (uint64_t i = 0; i < c->o->spp; ++i) {
    const double sx = ((double)x + rng_float(&rng)) / w;
    const double ty = ((double)y + rng_float(&rng)) / h;
    ov3 ro, rd;
    camera_ray(&c->cam, sx, ty, &rng, &ro, &rd);
    const ov3 col = trace_with(c->s, ro, rd, &rng, c->o->max_depth, (int)c->o->light_sampling, st, NULL, NULL);
    if (st) st->samples++;
    if (visfinite(col)) {
      sum = vadd(sum, col);
      const double lum = 0.2126 * col.x + 0.7152 * col.y + 0.0722 * col.z; /* light.zig:38-40 */
      lum2 += lum * lum;
    }
  }
  const ov3 px = vscale(sum, inv_spp);
  dst[0] = px.x;
  dst[1] = px.y;
  dst[2] = px.z;
  if (c->moments) c->moments[(dst - c->out) / 3] = lum2 * inv_spp;
}

static void stats_add(ostats* a, const ostats* b) {
  const uint64_t* src = (const uint64_t*)b;
  uint64_t* dst = (uint64_t*)a;
  for (size_t i = 0; i < sizeof(ostats) / sizeof(uint64_t); ++i) dst[i] += src[i];
}

static void* render_worker(void* arg) { /* Context.work, render.zig:113-119 */
  octx* c = (octx*)arg;
  ostats local;
  memset(&local, 0, sizeof local);
  ostats* st = c->stats ? &local : NULL;
  const uint64_t ts = c->o->tile_size;
  for (;;) {
    const uint64_t tile = atomic_fetch_add_explicit(&c->next_tile, 1, memory_order_relaxed);
    if (tile >= c->tile_count) break;
    if (c->pixels) { /* subset mode: tiles are runs of 64 listed pixels */
      const size_t b = (size_t)tile * 64, e = b + 64 < c->n_pixels ? b + 64 : c->n_pixels;
      for (size_t k = b; k < e; ++k) {
        const uint64_t p = c->pixels[k];
        render_pixel(c, p % c->o->width, p / c->o->width, c->out + 3 * k, st);
      }
      continue;
    }
    const uint64_t x0 = (tile % c->tiles_x) * ts, y0 = (tile / c->tiles_x) * ts; /* renderTile */
    const uint64_t x1 = x0 + ts < c->o->width ? x0 + ts : c->o->width;
    const uint64_t y1 = y0 + ts < c->o->height ? y0 + ts : c->o->height;
    for (uint64_t y = y0; y < y1; ++y)
      for (uint64_t x = x0; x < x1; ++x) render_pixel(c, x, y, c->out + 3 * (y * c->o->width + x), st);
  }
  if (c->stats) {
    pthread_mutex_lock(&c->stats_lock);
    stats_add(c->stats, &local);
    pthread_mutex_unlock(&c->stats_lock);
  }
  return NULL;
}

static int run_render(octx* c) { /* render.zig:169-178 */
  const uint64_t nthreads = c->o->threads < 1 ? 1 : c->o->threads;
  const uint64_t extra = (nthreads < c->tile_count ? nthreads : c->tile_count) - 1;
  pthread_t* th = (pthread_t*)malloc((extra ? extra : 1) * sizeof(pthread_t));
  if (!th) return -2;
  uint64_t spawned = 0;
  for (uint64_t i = 0; i < extra; ++i) {
    if (pthread_create(&th[i], NULL, render_worker, c) != 0) break;
    spawned++;
  }
  render_worker(c);
  for (uint64_t i = 0; i < spawned; ++i) pthread_join(th[i], NULL);
  free(th);
  return 0;
}

static int options_valid(const ooptions* o) { /* render.zig:153 */
  return !(o->width == 0 || o->height == 0 || o->spp == 0 || o->tile_size == 0);
}

int ozt_render(const oscene* s, const ooptions* o, double* out, ostats* stats) {
  if (!options_valid(o)) return -1;
  memset(out, 0, o->width * o->height * 3 * sizeof(double));
  octx c;
  memset(&c, 0, sizeof c);
  c.s = s;
  c.o = o;
  c.out = out;
  camera_init(&s->camera, (double)o->width / (double)o->height, &c.cam);
  c.tiles_x = (o->width + o->tile_size - 1) / o->tile_size;
  c.tile_count = c.tiles_x * ((o->height + o->tile_size - 1) / o->tile_size);
  atomic_init(&c.next_tile, 0);
  pthread_mutex_init(&c.stats_lock, NULL);
  if (stats) memset(stats, 0, sizeof *stats);
  c.stats = stats;
  const int rc = run_render(&c);
  pthread_mutex_destroy(&c.stats_lock);
  return rc;
}

int ozt_render_moments(const oscene* s, const ooptions* o, double* out, double* moments) {
  if (!options_valid(o)) return -1;
  memset(out, 0, o->width * o->height * 3 * sizeof(double));
  octx c;
  memset(&c, 0, sizeof c);
  c.s = s;
  c.o = o;
  c.out = out;
  c.moments = moments;
  camera_init(&s->camera, (double)o->width / (double)o->height, &c.cam);
  c.tiles_x = (o->width + o->tile_size - 1) / o->tile_size;
  c.tile_count = c.tiles_x * ((o->height + o->tile_size - 1) / o->tile_size);
  atomic_init(&c.next_tile, 0);
  pthread_mutex_init(&c.stats_lock, NULL);
  const int rc = run_render(&c);
  pthread_mutex_destroy(&c.stats_lock);
  return rc;
}

int ozt_render_pixels_moments(const oscene* s, const ooptions* o, const uint64_t* pixels, size_t n, double* out,
                              double* moments) {
  if (!options_valid(o)) return -1;
  octx c;
  memset(&c, 0, sizeof c);
  c.s = s;
  c.o = o;
  c.out = out;
  c.moments = moments;
  camera_init(&s->camera, (double)o->width / (double)o->height, &c.cam);
  c.pixels = pixels;
  c.n_pixels = n;
  c.tile_count = (n + 63) / 64;
  atomic_init(&c.next_tile, 0);
  pthread_mutex_init(&c.stats_lock, NULL);
  const int rc = c.tile_count ? run_render(&c) : 0;
  pthread_mutex_destroy(&c.stats_lock);
  return rc;
}

int ozt_render_pixels(const oscene* s, const ooptions* o, const uint64_t* pixels, size_t n, double* out,
                      ostats* stats) {
  if (!options_valid(o)) return -1;
  octx c;
  memset(&c, 0, sizeof c);
  c.s = s;
  c.o = o;
  c.out = out;
  camera_init(&s->camera, (double)o->width / (double)o->height, &c.cam);
  c.pixels = pixels;
  c.n_pixels = n;
  c.tile_count = (n + 63) / 64;
  atomic_init(&c.next_tile, 0);
  pthread_mutex_init(&c.stats_lock, NULL);
  if (stats) memset(stats, 0, sizeof *stats);
  c.stats = stats;
  const int rc = c.tile_count ? run_render(&c) : 0;
  pthread_mutex_destroy(&c.stats_lock);
  return rc;
}

int ozt_render_debug(const oscene* s, const ooptions* o, int32_t* first_prim, uint32_t* path_len) {
  if (!options_valid(o)) return -1;
  ocamera cam;
  camera_init(&s->camera, (double)o->width / (double)o->height, &cam);
  const double w = (double)o->width, h = (double)o->height;
  for (uint64_t y = 0; y < o->height; ++y)
    for (uint64_t x = 0; x < o->width; ++x) {
      const uint64_t p = y * o->width + x;
      orng rng = rng_for_stream(o->seed, p);
      const double sx = ((double)x + rng_float(&rng)) / w;
      const double ty = ((double)y + rng_float(&rng)) / h;
      ov3 ro, rd;
      camera_ray(&cam, sx, ty, &rng, &ro, &rd);
      trace_with(s, ro, rd, &rng, o->max_depth, (int)o->light_sampling, NULL, &first_prim[p], &path_len[p]);
    }
  return 0;
}

/* --------------------------------------------------------- Scene create --- */
int ozt_scene_create(const omaterial* mats, size_t n_mats, const oshape* shapes, size_t n_shapes,
                     const ocamera_config* cam, const obackground* bg, int build_bvh, oscene** out) {
  *out = NULL;
  for (size_t i = 0; i < n_shapes; ++i) {
    if (shapes[i].material >= n_mats || shapes[i].kind > O_PLANE) return -1;
  }
  oscene* s = (oscene*)calloc(1, sizeof(oscene));
  if (!s) return -2;
  s->mats = (omaterial*)malloc((n_mats ? n_mats : 1) * sizeof(omaterial));
  s->shapes = (oshape*)malloc((n_shapes ? n_shapes : 1) * sizeof(oshape));
  s->planes = (oshape*)malloc((n_shapes ? n_shapes : 1) * sizeof(oshape));
  if (!s->mats || !s->shapes || !s->planes) { ozt_scene_free(s); return -2; }
  if (n_mats) memcpy(s->mats, mats, n_mats * sizeof(omaterial));
  s->n_mats = n_mats;
  for (size_t i = 0; i < n_shapes; ++i) { /* Scene.add routes planes, scene.zig:71-78 */
    if (shapes[i].kind == O_PLANE) s->planes[s->n_planes++] = shapes[i];
    else s->shapes[s->n_shapes++] = shapes[i];
  }
  s->camera = *cam;
  s->background = *bg;
  if (build_bvh) { /* Scene.build, scene.zig:92-96 */
    int rc = bvh_build(s);
    if (rc == 0) rc = lights_build(s);
    if (rc != 0) { ozt_scene_free(s); return rc; }
    s->built = 1;
  }
  *out = s;
  return 0;
}

void ozt_scene_free(oscene* s) {
  if (!s) return;
  free(s->mats);
  free(s->shapes);
  free(s->planes);
  free(s->nodes);
  free(s->indices);
  free(s->lights);
  free(s->cdf);
  free(s);
}

size_t ozt_scene_bounded_count(const oscene* s) { return s->n_shapes; }
size_t ozt_scene_plane_count(const oscene* s) { return s->n_planes; }
size_t ozt_scene_node_count(const oscene* s) { return s->n_nodes; }
void ozt_scene_nodes(const oscene* s, onode* out) { if (s->n_nodes) memcpy(out, s->nodes, s->n_nodes * sizeof(onode)); }
void ozt_scene_indices(const oscene* s, uint32_t* out) {
  if (s->n_nodes) memcpy(out, s->indices, s->n_shapes * sizeof(uint32_t));
}
size_t ozt_scene_light_count(const oscene* s) { return s->n_lights; }
void ozt_scene_lights(const oscene* s, olight* out, double* cdf, double* total) {
  if (s->n_lights) {
    memcpy(out, s->lights, s->n_lights * sizeof(olight));
    memcpy(cdf, s->cdf, s->n_lights * sizeof(double));
  }
  *total = s->total;
}
static size_t depth_from(const oscene* s, uint32_t i) { /* bvh.zig:128-137 */
  const onode* n = &s->nodes[i];
  if (n->count > 0) return 1;
  const size_t a = depth_from(s, n->first), b = depth_from(s, n->first + 1);
  return 1 + (a > b ? a : b);
}
size_t ozt_bvh_depth(const oscene* s) { return s->n_nodes ? depth_from(s, 0) : 0; }

/* ------------------------------------------------------- Test entry points --- */
void ozt_trace_with(const oscene* s, const ov3* origin, const ov3* dir, uint64_t rng[4], uint64_t max_depth,
                    int light_sampling, ov3* out) {
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  *out = trace_with(s, *origin, *dir, &r, max_depth, light_sampling, NULL, NULL, NULL);
  memcpy(rng, r.s, sizeof r.s);
}
int ozt_scene_intersect(const oscene* s, const ov3* o, const ov3* d, double tmin, double tmax, ohit* out) {
  return scene_intersect(s, *o, *d, tmin, tmax, out, NULL);
}
int ozt_shape_intersect(const oshape* sh, const ov3* o, const ov3* d, double tmin, double tmax, ohit* out) {
  const int r = shape_intersect(sh, *o, *d, tmin, tmax, out, NULL);
  if (r) out->prim = 0;
  return r;
}
int ozt_intersect_all(const oshape* shapes, size_t n, const ov3* o, const ov3* d, double tmin, double tmax,
                      ohit* out) {
  return intersect_all(shapes, n, 0, *o, *d, tmin, tmax, out, NULL);
}
int ozt_lights_sample(const oscene* s, const ov3* origin, uint64_t rng[4], ov3* dir, double* distance, ov3* rad,
                      double* pdf) {
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  const int ok = lights_sample(s, *origin, &r, dir, distance, rad, pdf);
  memcpy(rng, r.s, sizeof r.s);
  return ok;
}
double ozt_lights_pdf_hit(const oscene* s, const ov3* origin, const ohit* hit) {
  return lights_pdf_hit(s, *origin, hit, NULL);
}
void ozt_material_emitted(const omaterial* m, const ohit* hit, ov3* out) { *out = material_emitted(m, hit); }
int ozt_material_scatter(const omaterial* m, const ov3* in_origin, const ov3* in_dir, const ohit* hit,
                         uint64_t rng[4], ov3* atten, ov3* out_origin, ov3* out_dir) {
  (void)in_origin;
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  const int ok = material_scatter(m, *in_dir, hit, &r, atten, out_origin, out_dir);
  memcpy(rng, r.s, sizeof r.s);
  return ok;
}
double ozt_schlick(double cosine, double eta) { return schlick(cosine, eta); }
void ozt_camera_init(const ocamera_config* cfg, double aspect, ocamera* out) { camera_init(cfg, aspect, out); }
void ozt_camera_ray(const ocamera* cam, double s, double t, uint64_t rng[4], ov3* origin, ov3* dir) {
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  camera_ray(cam, s, t, &r, origin, dir);
  memcpy(rng, r.s, sizeof r.s);
}
void ozt_background_radiance(const obackground* bg, const ov3* dir, ov3* out) {
  *out = background_radiance(bg, *dir);
}
void ozt_rng_init(uint64_t seed, uint64_t out[4]) { orng r = rng_init(seed); memcpy(out, r.s, sizeof r.s); }
void ozt_rng_for_stream(uint64_t seed, uint64_t stream, uint64_t out[4]) {
  orng r = rng_for_stream(seed, stream);
  memcpy(out, r.s, sizeof r.s);
}
void ozt_rng_next_n(uint64_t rng[4], size_t n, uint64_t* out) {
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  for (size_t i = 0; i < n; ++i) out[i] = rng_next(&r);
  memcpy(rng, r.s, sizeof r.s);
}
void ozt_rng_float_n(uint64_t rng[4], size_t n, double* out) {
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  for (size_t i = 0; i < n; ++i) out[i] = rng_float(&r);
  memcpy(rng, r.s, sizeof r.s);
}
uint64_t ozt_rng_below(uint64_t rng[4], uint64_t n) {
  orng r;
  memcpy(r.s, rng, sizeof r.s);
  const uint64_t v = rng_below(&r, n);
  memcpy(rng, r.s, sizeof r.s);
  return v;
}
#define RNG_WRAP(name, fn)                      \
  void name(uint64_t rng[4], ov3* out) {        \
    orng r;                                     \
    memcpy(r.s, rng, sizeof r.s);               \
    *out = fn(&r);                              \
    memcpy(rng, r.s, sizeof r.s);               \
  }
RNG_WRAP(ozt_rng_unit_vector, rng_unit_vector)
RNG_WRAP(ozt_rng_in_unit_sphere, rng_in_unit_sphere)
RNG_WRAP(ozt_rng_in_unit_disk, rng_in_unit_disk)
int ozt_aabb_hit(const ov3* bmin, const ov3* bmax, const ov3* o, const ov3* d, double tmin, double tmax, double* t) {
  return aabb_hit(bmin, bmax, *o, vinverse(*d), tmin, tmax, t);
}
/* image.zig:14-37 */
double ozt_tonemap(int kind, double c) {
  const double x = fmax(c, 0.0);
  if (kind == 0) return x;
  if (kind == 1) return x / (1.0 + x);
  return (x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14);
}
uint8_t ozt_encode(int kind, double gamma, double exposure, double linear) {
  const double v = isnan(linear) ? 0.0 : linear;
  const double mapped = fmax(0.0, fmin(ozt_tonemap(kind, v * exposure), 1.0));
  const double corrected = pow(mapped, 1.0 / gamma);
  return (uint8_t)round(fmax(0.0, fmin(corrected, 1.0)) * 255.0);
}
void ozt_sincos(double x, double* s, double* c) { zt_sincos(x, s, c); }
double ozt_pow5(double x) { return zt_pow5(x); }

/*
 * zt_device.cuh -- device functions of the radiance path (f64, sm_100a).
 *
 * Each function restates the reference routine named beside it with the same
 * IEEE-754 double operations in the same order.  The translation unit is
 * compiled with -fmad=false so no multiply-add is contracted, as in the
 * reference's strict-float Zig build; division and sqrt of doubles are the
 * correctly rounded CUDA defaults.  The result is a bit-exact device
 * restatement: same hits, same RNG draws, same radiance.
 */
#ifndef ZT_DEVICE_CUH
#define ZT_DEVICE_CUH

#include <stdint.h>

#include "zt_fpmath.h"
#include "zt_types.h"

namespace zt {

#define ZT_D __device__ __forceinline__

constexpr double kPi = 3.14159265358979323846;
constexpr double kRayEpsilon = 1e-4;  /* render.zig:26 */
constexpr uint64_t kRouletteDepth = 4; /* render.zig:28 */
constexpr int kStackSize = 66;         /* bvh.zig:87: max_depth + 2 */

/* ------------------------------------------------------------- Vec3 ---- */
/* src/vec.zig:5-125 */
struct dv3 { double x, y, z; };
ZT_D dv3 V(double x, double y, double z) { return dv3{x, y, z}; }
ZT_D dv3 L3(const double* p) { return dv3{p[0], p[1], p[2]}; }
ZT_D dv3 operator+(dv3 a, dv3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
ZT_D dv3 operator-(dv3 a, dv3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
ZT_D dv3 vmul(dv3 a, dv3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
ZT_D dv3 vscale(dv3 a, double s) { return V(a.x * s, a.y * s, a.z * s); }
ZT_D dv3 vdiv(dv3 a, double s) { return vscale(a, 1.0 / s); } /* vec.zig:37-39 */
ZT_D dv3 vneg(dv3 a) { return V(-a.x, -a.y, -a.z); }
ZT_D double vdot(dv3 a, dv3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
ZT_D dv3 vcross(dv3 a, dv3 b) {
  return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
ZT_D double vlen2(dv3 a) { return vdot(a, a); }
ZT_D double vlen(dv3 a) { return sqrt(vlen2(a)); }
ZT_D dv3 vnorm(dv3 a) { return vdiv(a, vlen(a)); }
ZT_D dv3 vlerp(dv3 a, dv3 b, double t) { return vscale(a, 1.0 - t) + vscale(b, t); }
ZT_D double vmaxc(dv3 a) { return fmax(a.x, fmax(a.y, a.z)); }
/* std.math.clamp(x, 0, 1) = @max(0, @min(x, 1)): a NaN x gives 1.  The NaN
 * case is spelled out because nvcc may turn fmax(0, fmin(x, 1)) into a
 * saturating operation, which maps NaN to 0 (measured on sm_100a). */
ZT_D double clamp01(double x) { return isnan(x) ? 1.0 : fmax(0.0, fmin(x, 1.0)); }
ZT_D bool vnear_zero(dv3 a) {
  const double eps = 1e-8;
  return fabs(a.x) < eps && fabs(a.y) < eps && fabs(a.z) < eps;
}
ZT_D bool visfinite(dv3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
ZT_D dv3 vreflect(dv3 v, dv3 n) { return v - vscale(n, 2.0 * vdot(v, n)); }
ZT_D dv3 vrefract(dv3 uv, dv3 n, double eta) { /* vec.zig:119-124 */
  const double cos_theta = fmin(vdot(vneg(uv), n), 1.0);
  const dv3 r_perp = vscale(uv + vscale(n, cos_theta), eta);
  const dv3 r_par = vscale(n, -sqrt(fabs(1.0 - vlen2(r_perp))));
  return r_perp + r_par;
}

/* -------------------------------------------------------------- Rng ---- */
/* src/rng.zig:10-88 */
struct Rng { uint64_t s0, s1, s2, s3; };

ZT_D uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
ZT_D uint64_t splitmix64(uint64_t& state) {
  state += 0x9E3779B97F4A7C15ULL;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
ZT_D Rng rng_for_stream(uint64_t seed, uint64_t stream) { /* rng.zig:22-25 */
  uint64_t sm = seed ^ (stream * 0x9E3779B97F4A7C15ULL);
  uint64_t s2 = splitmix64(sm);
  Rng r;
  r.s0 = splitmix64(s2);
  r.s1 = splitmix64(s2);
  r.s2 = splitmix64(s2);
  r.s3 = splitmix64(s2);
  return r;
}
ZT_D uint64_t rng_next(Rng& r) { /* rng.zig:27-38, xoshiro256++ */
  const uint64_t result = rotl64(r.s0 + r.s3, 23) + r.s0;
  const uint64_t t = r.s1 << 17;
  r.s2 ^= r.s0;
  r.s3 ^= r.s1;
  r.s1 ^= r.s2;
  r.s0 ^= r.s3;
  r.s2 ^= t;
  r.s3 = rotl64(r.s3, 45);
  return result;
}
ZT_D double rng_float(Rng& r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }
ZT_D double rng_range(Rng& r, double lo, double hi) { return lo + (hi - lo) * rng_float(r); }
ZT_D dv3 rng_unit_vector(Rng& r) { /* rng.zig:58-63 */
  const double z = rng_range(r, -1.0, 1.0);
  const double phi = rng_range(r, 0.0, 2.0 * kPi);
  const double rr = sqrt(fmax(0.0, 1.0 - z * z));
  double s, c;
  zt_sincos(phi, &s, &c);
  return V(rr * c, rr * s, z);
}
ZT_D dv3 rng_in_unit_disk(Rng& r) { /* rng.zig:74-79 */
  for (;;) {
    const double x = rng_range(r, -1, 1);
    const double y = rng_range(r, -1, 1);
    if (x * x + y * y + 0.0 * 0.0 < 1.0) return V(x, y, 0);
  }
}

/* -------------------------------------------------------------- Hit ---- */
/* src/geometry.zig:11-30; prim is instrumentation only. */
struct Hit {
  double t;
  dv3 point, normal;
  uint32_t front_face, material;
  int32_t prim;
};

ZT_D void hit_make(dv3 o, dv3 d, double t, dv3 outward, uint32_t mat, Hit& h) {
  const bool front = vdot(d, outward) < 0;
  h.t = t;
  h.point = o + vscale(d, t); /* Ray.at, ray.zig:12-14 */
  h.normal = front ? outward : vneg(outward);
  h.front_face = front;
  h.material = mat;
}

/* Sphere.intersect, geometry.zig:37-52.  Returns the root t or a value
 * outside the range; the hit record is built only for the closest hit. */
ZT_D bool sphere_t(dv3 center, double radius, dv3 o, dv3 d, double tmin, double tmax, double& tout) {
  const dv3 oc = center - o;
  const double a = vlen2(d);
  const double h = vdot(d, oc);
  const double c = vlen2(oc) - radius * radius;
  const double disc = h * h - a * c;
  if (disc < 0) return false;
  const double sq = sqrt(disc);
  double t = (h - sq) / a;
  if (t <= tmin || t >= tmax) {
    t = (h + sq) / a;
    if (t <= tmin || t >= tmax) return false;
  }
  tout = t;
  return true;
}
ZT_D void sphere_hit(dv3 center, double radius, uint32_t mat, dv3 o, dv3 d, double t, Hit& h) {
  const dv3 outward = vdiv((o + vscale(d, t)) - center, radius);
  hit_make(o, d, t, outward, mat, h);
}

/* Moller-Trumbore, geometry.zig:83-99, with e1/e2 precomputed. */
ZT_D bool triangle_t(dv3 v0, dv3 e1, dv3 e2, dv3 o, dv3 d, double tmin, double tmax, double& tout) {
  const dv3 p = vcross(d, e2);
  const double det = vdot(e1, p);
  if (fabs(det) < 1e-12) return false;
  const double inv_det = 1.0 / det;
  const dv3 s = o - v0;
  const double u = vdot(s, p) * inv_det;
  if (u < 0 || u > 1) return false;
  const dv3 q = vcross(s, e1);
  const double v = vdot(d, q) * inv_det;
  if (v < 0 || u + v > 1) return false;
  const double t = vdot(e2, q) * inv_det;
  if (t <= tmin || t >= tmax) return false;
  tout = t;
  return true;
}
ZT_D void triangle_hit(dv3 e1, dv3 e2, uint32_t mat, dv3 o, dv3 d, double t, Hit& h) {
  hit_make(o, d, t, vnorm(vcross(e1, e2)), mat, h);
}

/* Plane.intersect, geometry.zig:67-73. */
ZT_D bool plane_t(dv3 point, dv3 normal, dv3 o, dv3 d, double tmin, double tmax, double& tout) {
  const double denom = vdot(normal, d);
  if (fabs(denom) < 1e-12) return false;
  const double t = vdot(point - o, normal) / denom;
  if (t <= tmin || t >= tmax) return false;
  tout = t;
  return true;
}

/* A primitive of the BVH: a sphere or a triangle (planes are unbounded and
 * never enter the tree, scene.zig:84-96), so the closest-hit leaf loops
 * carry no plane code: on the 256 sphere-field batch 52.6 against 58.6 ms
 * per launch.  The any-hit walks keep the general prim_t below, measured 1%
 * faster on the 1M-triangle terrain (where shadow rays are half the frame)
 * and the same elsewhere; both give the same answer for every primitive of
 * the tree. */
ZT_D bool bounded_t(const DPrim& pg, dv3 o, dv3 d, double tmin, double tmax, double& t) {
  /* five 16-byte read-only loads of the 80-byte record */
  const double2* q = reinterpret_cast<const double2*>(&pg);
  const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3), q4 = __ldg(q + 4);
  const uint32_t kind = (uint32_t)((unsigned long long)__double_as_longlong(q4.y) >> 32); /* material, kind */
  if (kind == kTriangle)
    return triangle_t(V(q0.x, q0.y, q1.x), V(q1.y, q2.x, q2.y), V(q3.x, q3.y, q4.x), o, d, tmin, tmax, t);
  return sphere_t(V(q0.x, q0.y, q1.x), q1.y, o, d, tmin, tmax, t);
}
/* Any primitive kind (the any-hit walks' leaf and plane loops). */
ZT_D bool prim_t(const DPrim& pg, dv3 o, dv3 d, double tmin, double tmax, double& t) {
  /* five 16-byte read-only loads of the 80-byte record */
  const double2* q = reinterpret_cast<const double2*>(&pg);
  const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2), q3 = __ldg(q + 3), q4 = __ldg(q + 4);
  DPrim p;
  p.a[0] = q0.x; p.a[1] = q0.y; p.a[2] = q1.x; p.a[3] = q1.y; p.a[4] = q2.x;
  p.a[5] = q2.y; p.a[6] = q3.x; p.a[7] = q3.y; p.a[8] = q4.x;
  p.kind = (uint32_t)((unsigned long long)__double_as_longlong(q4.y) >> 32); /* material, kind */
  if (p.kind == kTriangle) return triangle_t(L3(p.a), L3(p.a + 3), L3(p.a + 6), o, d, tmin, tmax, t);
  if (p.kind == kSphere) return sphere_t(L3(p.a), p.a[3], o, d, tmin, tmax, t);
  return plane_t(L3(p.a), L3(p.a + 3), o, d, tmin, tmax, t);
}
/* One of the scene's unbounded planes (point, normal). */
ZT_D bool plane_prim_t(const DPrim& pg, dv3 o, dv3 d, double tmin, double tmax, double& t) {
  const double2* q = reinterpret_cast<const double2*>(&pg);
  const double2 q0 = __ldg(q), q1 = __ldg(q + 1), q2 = __ldg(q + 2);
  return plane_t(V(q0.x, q0.y, q1.x), V(q1.y, q2.x, q2.y), o, d, tmin, tmax, t);
}
ZT_D void bounded_hit(const DPrim& p, dv3 o, dv3 d, double t, Hit& h) {
  if (p.kind == kTriangle) triangle_hit(L3(p.a + 3), L3(p.a + 6), p.material, o, d, t, h);
  else sphere_hit(L3(p.a), p.a[3], p.material, o, d, t, h);
}

/* --------------------------------------------------------- Traversal ---- */
/* Slab test of one box, aabb.zig:68-83.  The reference returns early once
 * hi < lo; lo only grows and hi only shrinks afterwards, so testing once at
 * the end is the same predicate.  The updates keep the reference's compares
 * (a NaN plane distance, 0 * inf, leaves lo and hi unchanged): written as
 * compare-and-select they measured faster than f64 fmax/fmin. */
ZT_D bool slab(const double* lo3, const double* hi3, dv3 o, dv3 inv, double tmin, double tmax, double& tout) {
  double lo = tmin, hi = tmax;
  {
    double t0 = (lo3[0] - o.x) * inv.x, t1 = (hi3[0] - o.x) * inv.x;
    const bool sw = inv.x < 0;
    const double n = sw ? t1 : t0, f = sw ? t0 : t1;
    lo = n > lo ? n : lo;
    hi = f < hi ? f : hi;
  }
  {
    double t0 = (lo3[1] - o.y) * inv.y, t1 = (hi3[1] - o.y) * inv.y;
    const bool sw = inv.y < 0;
    const double n = sw ? t1 : t0, f = sw ? t0 : t1;
    lo = n > lo ? n : lo;
    hi = f < hi ? f : hi;
  }
  {
    double t0 = (lo3[2] - o.z) * inv.z, t1 = (hi3[2] - o.z) * inv.z;
    const bool sw = inv.z < 0;
    const double n = sw ? t1 : t0, f = sw ? t0 : t1;
    lo = n > lo ? n : lo;
    hi = f < hi ? f : hi;
  }
  tout = lo;
  return !(hi < lo);
}

struct StackEntry { uint32_t first, count; double t; };

/* Scene.intersect (scene.zig:108-116): Bvh.intersect (bvh.zig:80-126) with
 * the same nearest-first order, `tl <= tr` tie-break and `entry.t > closest`
 * pruning, then the unbounded planes up to the BVH hit.  any_hit = true stops
 * at the first primitive hit: the traversal up to that point is identical,
 * so whether a hit exists is the same answer the reference's closest-hit
 * query gives to `!= null` (render.zig:51). */
ZT_D int32_t scene_query_rt(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax, bool any_hit,
                            double& t_out);
template <bool kAnyHit>
ZT_D int32_t scene_query(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax, double& t_out) {
  return scene_query_rt(sc, o, d, tmin, tmax, kAnyHit, t_out);
}

/* The hit record of a query result (prim code k at distance t). */
ZT_D void hit_from(const DevScene& sc, int32_t k, dv3 o, dv3 d, double t, Hit& out) {
  if (k >= 0) {
    bounded_hit(sc.prims[k], o, d, t, out);
    out.prim = sc.prim_ids[k];
  } else {
    const int32_t pi = -2 - k;
    const DPrim& pl = sc.planes[pi];
    hit_make(o, d, t, L3(pl.a + 3), pl.material, out);
    out.prim = (int32_t)sc.n_prims + pi;
  }
}



/* Returns the prim code of the closest hit (>= 0: prims[k]; <= -2:
 * planes[-2 - k]; -1: no hit) and its distance.  any_hit is a run-time flag
 * so that lanes with closest-hit and any-hit queries share one traversal. */
ZT_D int32_t scene_query_rt(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax, bool kAnyHit,
                            double& t_out) {
  double closest = tmax;
  int32_t best_k = -1;  /* >= 0: prims[best_k]; <= -2: planes[-2 - best_k] */
  double t;
  const dv3 inv = V(1.0 / d.x, 1.0 / d.y, 1.0 / d.z); /* aabb.zig:86-88 */
  if (sc.has_root && slab(sc.root_lo, sc.root_hi, o, inv, tmin, closest, t)) {
    /* Nearest-first stack traversal, bvh.zig:94-124.  The nearer child of a
     * two-hit node stays in registers as the next entry instead of being
     * pushed and popped at once: the same visiting order and pop check. */
    StackEntry stack[kStackSize];
    StackEntry e;
    e.first = sc.root_first;
    e.count = sc.root_count;
    e.t = t;
    bool have = true;
    int sp = 0;
    for (;;) {
      if (!have) {
        if (sp == 0) break;
        e = stack[--sp];
      }
      have = false;
      if (e.t > closest) continue; /* bvh.zig:97 */
      if (e.count > 0) {
        for (uint32_t k = e.first; k < e.first + e.count; ++k) {
          double th;
          if (bounded_t(sc.prims[k], o, d, tmin, closest, th)) {
            closest = th;
            best_k = (int32_t)k;
            if (kAnyHit) { t_out = th; return best_k; }
          }
        }
        continue;
      }
      const double2* rec = reinterpret_cast<const double2*>(sc.pairs + e.first);
      const double2 a0 = __ldg(rec + 0), a1 = __ldg(rec + 1), a2 = __ldg(rec + 2);
      const double2 b0 = __ldg(rec + 3), b1 = __ldg(rec + 4), b2 = __ldg(rec + 5);
      const uint4 pc = __ldg(reinterpret_cast<const uint4*>(rec + 6));
      /* lo[0] = a0.x a0.y a1.x, lo[1] = a1.y a2.x a2.y, hi[0] = b0.x b0.y b1.x, hi[1] = b1.y b2.x b2.y */
      const double lo0[3] = {a0.x, a0.y, a1.x}, lo1[3] = {a1.y, a2.x, a2.y};
      const double hi0[3] = {b0.x, b0.y, b1.x}, hi1[3] = {b1.y, b2.x, b2.y};
      double tl, tr;
      const bool hl = slab(lo0, hi0, o, inv, tmin, closest, tl);
      const bool hr = slab(lo1, hi1, o, inv, tmin, closest, tr);
      if (hl && hr) { /* push the farther child; the nearer one is popped next (bvh.zig:111-116) */
        const bool near_left = tl <= tr;
        stack[sp].first = near_left ? pc.y : pc.x;
        stack[sp].count = near_left ? pc.w : pc.z;
        stack[sp].t = near_left ? tr : tl;
        sp += 1;
        e.first = near_left ? pc.x : pc.y;
        e.count = near_left ? pc.z : pc.w;
        e.t = near_left ? tl : tr;
        have = true;
      } else if (hl || hr) {
        e.first = hl ? pc.x : pc.y;
        e.count = hl ? pc.z : pc.w;
        e.t = hl ? tl : tr;
        have = true;
      }
    }
  }
  /* intersectAll(planes, r, t_min, limit), geometry.zig:129-139 */
  for (uint32_t i = 0; i < sc.n_planes; ++i) {
    double th;
    if (plane_prim_t(sc.planes[i], o, d, tmin, closest, th)) {
      closest = th;
      best_k = -2 - (int32_t)i;
      if (kAnyHit) { t_out = th; return best_k; }
    }
  }
  t_out = closest;
  return best_k;
}


/* Shadow query: whether any primitive is hit in (tmin, tmax)
 * (`scene.intersect(...) != null`, render.zig:51).  The answer does not
 * depend on the order of the BVH walk: until its first hit the reference's
 * walk prunes with the fixed tmax, so it reaches a hit iff some leaf whose
 * box the ray overlaps below tmax holds a primitive hit in (tmin, tmax) --
 * a property of the set of such leaves, not of the order they are visited
 * in.  Every stack entry was pushed with t <= tmax, so the entry distance
 * and the pop check are dropped (the stack holds first, count) and the walk
 * stops at the first hit.  It visits the farther child first: occluders of
 * rays leaving a surface lie away from the origin more often than near it
 * (measured 3.7% faster on the 1M-triangle scene than nearest first). */
ZT_D bool scene_occluded(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax) {
  const dv3 inv = V(1.0 / d.x, 1.0 / d.y, 1.0 / d.z); /* aabb.zig:86-88 */
  double t;
  if (sc.has_root && slab(sc.root_lo, sc.root_hi, o, inv, tmin, tmax, t)) {
    uint2 stack[kStackSize];
    uint32_t first = sc.root_first, count = sc.root_count;
    bool have = true;
    int sp = 0;
    for (;;) {
      if (!have) {
        if (sp == 0) break;
        const uint2 e = stack[--sp];
        first = e.x;
        count = e.y;
      }
      have = false;
      if (count > 0) {
        for (uint32_t k = first; k < first + count; ++k) {
          double th;
          if (prim_t(sc.prims[k], o, d, tmin, tmax, th)) return true;
        }
        continue;
      }
      const double2* rec = reinterpret_cast<const double2*>(sc.pairs + first);
      const double2 a0 = __ldg(rec + 0), a1 = __ldg(rec + 1), a2 = __ldg(rec + 2);
      const double2 b0 = __ldg(rec + 3), b1 = __ldg(rec + 4), b2 = __ldg(rec + 5);
      const uint4 pc = __ldg(reinterpret_cast<const uint4*>(rec + 6));
      const double lo0[3] = {a0.x, a0.y, a1.x}, lo1[3] = {a1.y, a2.x, a2.y};
      const double hi0[3] = {b0.x, b0.y, b1.x}, hi1[3] = {b1.y, b2.x, b2.y};
      double tl, tr;
      const bool hl = slab(lo0, hi0, o, inv, tmin, tmax, tl);
      const bool hr = slab(lo1, hi1, o, inv, tmin, tmax, tr);
      if (hl && hr) {
        const bool left_first = tl > tr; /* the farther child first */
        stack[sp] = make_uint2(left_first ? pc.y : pc.x, left_first ? pc.w : pc.z);
        sp += 1;
        first = left_first ? pc.x : pc.y;
        count = left_first ? pc.z : pc.w;
        have = true;
      } else if (hl || hr) {
        first = hl ? pc.x : pc.y;
        count = hl ? pc.z : pc.w;
        have = true;
      }
    }
  }
  for (uint32_t i = 0; i < sc.n_planes; ++i) { /* geometry.zig:129-139 */
    double th;
    if (prim_t(sc.planes[i], o, d, tmin, tmax, th)) return true;
  }
  return false;
}

}  // namespace zt

#include "zt_fast.cuh"

namespace zt {

/* Closest or any hit with the hit record (kAnyHit: t only).  kFast walks
 * the float records (zt_fast.cuh) for closest-hit queries. */
template <bool kAnyHit, bool kFast = false>
ZT_D bool scene_intersect(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax, Hit& out) {
  double t;
  const int32_t k = (kFast && !kAnyHit) ? scene_query_fast(sc, o, d, tmin, tmax, t)
                                        : scene_query<kAnyHit>(sc, o, d, tmin, tmax, t);
  if (k == -1) return false;
  out.t = t;
  if (!kAnyHit) hit_from(sc, k, o, d, t, out);
  return true;
}

/* ---------------------------------------------------------- Material ---- */
/* src/material.zig */
ZT_D double schlick(double cosine, double eta) { /* material.zig:66-70 */
  double r0 = (1.0 - eta) / (1.0 + eta);
  r0 *= r0;
  return r0 + (1.0 - r0) * zt_pow5(1.0 - cosine);
}

/* Material.scatter, material.zig:34-62. */
ZT_D bool material_scatter(const DMat& m, dv3 in_dir, const Hit& h, Rng& rng, dv3& atten, dv3& out_d) {
  /* One call site each for the unit-vector draw (a Lambertian bounce and a
   * fuzzy metal's perturbation, the only draws of those branches) and for
   * normalising the incoming direction (metal and dielectric): the same
   * draws in the same order, half the inlined code. */
  const bool lambertian = m.kind == kLambertian, metal = m.kind == kMetal;
  dv3 uv = V(0, 0, 0), unit = V(0, 0, 0);
  if (lambertian || (metal && m.param > 0)) uv = rng_unit_vector(rng);
  if (metal || m.kind == kDielectric) unit = vnorm(in_dir);
  if (lambertian) {
    dv3 dir = h.normal + uv;
    if (vnear_zero(dir)) dir = h.normal;
    atten = L3(m.color);
    out_d = vnorm(dir);
    return true;
  }
  if (metal) {
    dv3 dir = vreflect(unit, h.normal);
    if (m.param > 0) dir = vnorm(dir + vscale(uv, m.param));
    if (vdot(dir, h.normal) <= 0) return false;
    atten = L3(m.color);
    out_d = dir;
    return true;
  }
  if (m.kind == kDielectric) {
    const double eta = h.front_face ? 1.0 / m.param : m.param;
    const double cos_theta = fmin(vdot(vneg(unit), h.normal), 1.0);
    const double sin_theta = sqrt(fmax(0.0, 1.0 - cos_theta * cos_theta));
    const bool cannot_refract = eta * sin_theta > 1.0;
    /* `or` short-circuits (material.zig:54): no draw under TIR */
    if (cannot_refract || schlick(cos_theta, eta) > rng_float(rng)) out_d = vreflect(unit, h.normal);
    else out_d = vrefract(unit, h.normal, eta);
    atten = V(1, 1, 1);
    return true;
  }
  return false;
}

/* ------------------------------------------------------------- Light ---- */
/* src/light.zig */
ZT_D bool sphere_outside(dv3 center, double radius, dv3 origin) { /* light.zig:47-50 */
  return vlen(center - origin) > fabs(radius) * (1 + 1e-9);
}

/* The sphere-light half of Lights.sample (light.zig:143-163).  Light
 * sampling takes it outlined (sphere_light_sample below) in every kernel but
 * the fast-walk instances: the scenes measured have quad lights only, and
 * keeping this code out of the kernels' bodies shortens the instruction
 * stream the warps fetch (Cornell box 530 -> 581 Msamples/s, path-replay
 * backward 54.3 -> 50.7 ms), while the 64-register fast instances measured
 * 4% slower with the call in their body (1M triangles 1025 -> 982). */
ZT_D bool sphere_light_sample_impl(const DLight& L, double select, dv3 origin, Rng& rng, dv3& odir,
                                   double& odist, dv3& orad, double& opdf) {
  const dv3 center = L3(L.v);
  const double radius = L.v[3];
  if (!sphere_outside(center, radius, origin)) return false;
  const dv3 axis = center - origin;
  const double d2 = vlen2(axis);
  const dv3 w = vscale(axis, 1 / sqrt(d2));
  const double cos_max = sqrt(fmax(0.0, 1 - radius * radius / d2));
  const double cos_t = 1 - rng_float(rng) * (1 - cos_max);
  const double sin_t = sqrt(fmax(0.0, 1 - cos_t * cos_t));
  const double phi = 2 * kPi * rng_float(rng);
  /* basis, light.zig:53-57 */
  const dv3 a = fabs(w.x) > 0.9 ? V(0, 1, 0) : V(1, 0, 0);
  const dv3 bv = vnorm(vcross(w, a));
  const dv3 bu = vcross(bv, w);
  double sphi, cphi;
  zt_sincos(phi, &sphi, &cphi);
  const dv3 dir = vnorm((vscale(bu, sin_t * cphi) + vscale(bv, sin_t * sphi)) + vscale(w, cos_t));
  double th;
  if (!sphere_t(center, radius, origin, dir, 0, INFINITY, th)) return false;
  /* hit.front_face of the sphere hit at th */
  const dv3 outward = vdiv((origin + vscale(dir, th)) - center, radius);
  if (!(vdot(dir, outward) < 0)) return false;
  odir = dir;
  odist = th;
  orad = L3(L.radiance);
  opdf = select / (2 * kPi * (1 - cos_max));
  return true;
}
__device__ __noinline__ bool sphere_light_sample(const DLight& L, double select, dv3 origin, Rng& rng, dv3& odir,
                                                 double& odist, dv3& orad, double& opdf) {
  return sphere_light_sample_impl(L, select, origin, rng, odir, odist, orad, opdf);
}

/* The sphere-light term of Lights.pdfHit (light.zig:186-193): select /
 * (2 pi (1 - cos_max)) where the ray from origin along dir reaches the front
 * of the sphere at distance dist, else 0.  Inline or outlined as the
 * sampling half above. */
ZT_D double sphere_light_pdf_impl(const DLight& L, double select, dv3 origin, dv3 dir, double dist) {
  const dv3 center = L3(L.v);
  const double radius = L.v[3];
  if (!sphere_outside(center, radius, origin)) return 0;
  double th;
  if (!sphere_t(center, radius, origin, dir, 1e-9, INFINITY, th)) return 0;
  const dv3 outward = vdiv((origin + vscale(dir, th)) - center, radius);
  const bool front = vdot(dir, outward) < 0;
  if (fabs(th - dist) > 1e-6 * dist || !front) return 0;
  const double d2 = vlen2(center - origin);
  const double cos_max = sqrt(fmax(0.0, 1 - radius * radius / d2));
  return select / (2 * kPi * (1 - cos_max));
}
__device__ __noinline__ double sphere_light_pdf(const DLight& L, double select, dv3 origin, dv3 dir, double dist) {
  return sphere_light_pdf_impl(L, select, origin, dir, dist);
}

/* Lights.sample, light.zig:120-166.  kInlineSphere: the sphere-light code
 * inline (the fast-walk instances) rather than called. */
template <bool kInlineSphere = false>
ZT_D bool lights_sample(const DevScene& sc, dv3 origin, Rng& rng, dv3& odir, double& odist, dv3& orad,
                        double& opdf, uint32_t* picked = nullptr) {
  if (sc.n_lights == 0) return false;
  /* pick, light.zig:106-115 */
  const double x = rng_float(rng) * sc.total;
  uint32_t lo = 0, hi = sc.n_lights - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) / 2;
    if (sc.cdf[mid] > x) hi = mid;
    else lo = mid + 1;
  }
  const DLight& L = sc.lights[lo];
  if (picked) *picked = lo;
  const double select = L.weight / sc.total;
  if (L.kind == kTriangle) {
    const dv3 v0 = L3(L.v), v1 = L3(L.v + 3), v2 = L3(L.v + 6);
    const double su = sqrt(rng_float(rng));
    const double b2 = rng_float(rng);
    const dv3 p = (vscale(v0, 1 - su) + vscale(v1, su * (1 - b2))) + vscale(v2, su * b2);
    const dv3 to = p - origin;
    const double dist = vlen(to);
    if (dist < 1e-9) return false;
    const dv3 dir = vscale(to, 1 / dist);
    const double cos_l = -vdot(dir, L3(L.normal));
    if (cos_l <= 1e-9) return false;
    odir = dir;
    odist = dist;
    orad = L3(L.radiance);
    opdf = select * dist * dist / (cos_l * L.area);
    return true;
  }
  if (kInlineSphere) return sphere_light_sample_impl(L, select, origin, rng, odir, odist, orad, opdf);
  return sphere_light_sample(L, select, origin, rng, odir, odist, orad, opdf);
}

/* Lights.pdfHit, light.zig:171-198; kInlineSphere as for lights_sample. */
template <bool kInlineSphere = false>
ZT_D double lights_pdf_hit(const DevScene& sc, dv3 origin, dv3 hit_point) {
  const dv3 to = hit_point - origin;
  const double dist = vlen(to);
  if (dist < 1e-9) return 0;
  const dv3 dir = vscale(to, 1 / dist);
  double pdf = 0;
  for (uint32_t i = 0; i < sc.n_lights; ++i) {
    const DLight& L = sc.lights[i];
    const double select = L.weight / sc.total;
    if (L.kind == kTriangle) {
      const dv3 v0 = L3(L.v);
      const dv3 e1 = L3(L.v + 3) - v0, e2 = L3(L.v + 6) - v0;
      double th;
      if (!triangle_t(v0, e1, e2, origin, dir, 1e-9, INFINITY, th)) continue;
      /* Hit.make with the outward normal normalize(e1 x e2) */
      const dv3 outward = vnorm(vcross(e1, e2));
      const bool front = vdot(dir, outward) < 0;
      if (fabs(th - dist) > 1e-6 * dist || !front) continue;
      const dv3 n = front ? outward : vneg(outward);
      pdf += select * dist * dist / (-vdot(dir, n) * L.area);
    } else {
      pdf += kInlineSphere ? sphere_light_pdf_impl(L, select, origin, dir, dist)
                           : sphere_light_pdf(L, select, origin, dir, dist);
    }
  }
  return pdf;
}

/* ----------------------------------------------------------- Camera ---- */
ZT_D void camera_ray(const DCamera& c, double s, double t, Rng& rng, dv3& ro, dv3& rd) { /* camera.zig:59-67 */
  dv3 origin = L3(c.origin);
  if (c.lens_radius > 0) {
    const dv3 p = rng_in_unit_disk(rng);
    const dv3 d = vscale(p, c.lens_radius);
    origin = (origin + vscale(L3(c.u), d.x)) + vscale(L3(c.v), d.y);
  }
  const dv3 target = (L3(c.upper_left) + vscale(L3(c.horizontal), s)) + vscale(L3(c.vertical), t);
  ro = origin;
  rd = vnorm(target - origin);
}

ZT_D dv3 background_radiance(const DBackground& bg, dv3 dir) { /* scene.zig:20-28 */
  if (bg.kind == 0) return L3(bg.a);
  const double t = clamp01(vnorm(dir).y);
  return vlerp(L3(bg.a), L3(bg.b), t);
}

/* -------------------------------------------------------- Integrator ---- */
ZT_D double power_weight(double a, double b) { /* render.zig:38-41 */
  const double a2 = a * a;
  return a2 / (a2 + b * b);
}

/* directLight, render.zig:46-56 (shadow ray as an any-hit query; kFast
 * walks the float records). */
template <bool kFast = false>
ZT_D dv3 direct_light(const DevScene& sc, dv3 albedo, const Hit& hit, Rng& rng) {
  dv3 ldir, lrad;
  double ldist, lpdf;
  if (!lights_sample<kFast>(sc, hit.point, rng, ldir, ldist, lrad, lpdf)) return V(0, 0, 0);
  const double cos_s = vdot(hit.normal, ldir);
  if (cos_s <= 0 || !(lpdf > 0)) return V(0, 0, 0);
  const double shadow_tmax = ldist * (1 - 1e-6);
  if (kFast ? scene_occluded_fast(sc, hit.point, ldir, kRayEpsilon, shadow_tmax)
            : scene_occluded(sc, hit.point, ldir, kRayEpsilon, shadow_tmax))
    return V(0, 0, 0);
  const double bsdf_pdf = cos_s / kPi;
  const double scale = cos_s / (kPi * lpdf) * power_weight(lpdf, bsdf_pdf);
  return vscale(vmul(albedo, lrad), scale);
}

/* traceWith, render.zig:61-102.  kNee = false compiles light sampling out
 * (for scenes where use_nee is false: no lights or light_sampling off); the
 * path is then the reference's use_nee = false path, draw for draw. */
struct TraceAux { int32_t first_prim; uint32_t path_len; };

template <bool kAux, bool kNee = true, bool kFast = false>
ZT_D dv3 trace_with(const DevScene& sc, dv3 ro, dv3 rd, Rng& rng, uint64_t max_depth, bool use_nee_arg,
                    TraceAux* aux) {
  const bool use_nee = kNee && use_nee_arg;
  /* The reference's prev_origin (render.zig:66-70) is read only when
   * prev_pdf > 0, i.e. after a bounce, where it always equals the current
   * ray's origin ro: ro stands in for it and keeps three doubles out of the
   * registers that stay live across every traversal. */
  dv3 radiance = V(0, 0, 0), throughput = V(1, 1, 1);
  double prev_pdf = 0;
  uint32_t n_ext = 0;
  if (kAux) aux->first_prim = -1;
  for (uint64_t depth = 0; depth < max_depth; ++depth) {
    Hit hit;
    if (kAux) n_ext++;
    if (!scene_intersect<false, kFast>(sc, ro, rd, kRayEpsilon, INFINITY, hit)) {
      if (kAux) aux->path_len = n_ext;
      return radiance + vmul(throughput, background_radiance(sc.bg, rd));
    }
    if (kAux && depth == 0) aux->first_prim = hit.prim;
    const DMat& mat = sc.mats[hit.material];
    /* Material.emitted, material.zig:26-32 */
    const dv3 le = (mat.kind == kEmissive && hit.front_face) ? L3(mat.color) : V(0, 0, 0);
    if (vmaxc(le) > 0) {
      const double w = prev_pdf > 0 ? power_weight(prev_pdf, lights_pdf_hit<kFast>(sc, ro, hit.point)) : 1.0;
      radiance = radiance + vscale(vmul(throughput, le), w);
    }
    if (mat.kind == kLambertian && use_nee)
      radiance = radiance + vmul(throughput, direct_light<kFast>(sc, L3(mat.color), hit, rng));
    dv3 atten, sd;
    if (!material_scatter(mat, rd, hit, rng, atten, sd)) break;
    throughput = vmul(throughput, atten);
    prev_pdf = (use_nee && mat.kind == kLambertian) ? fmax(vdot(sd, hit.normal), 0.0) / kPi : 0;
    ro = hit.point;
    rd = sd;
    if (depth + 1 >= kRouletteDepth) {
      const double p = fmin(vmaxc(throughput), 0.95);
      if (p <= 0 || rng_float(rng) >= p) break;
      throughput = vdiv(throughput, p);
    }
  }
  if (kAux) aux->path_len = n_ext;
  return radiance;
}

}  // namespace zt

#endif

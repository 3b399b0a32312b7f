/*
 * zt_fast.cuh -- the fast traversal: the reference's BVH walk
 * (src/bvh.zig:80-126) over conservative single-precision boxes.
 *
 * The box tests of the f64 walk are three quarters of its arithmetic and run
 * on the FP64 pipe, which issues a warp instruction every other cycle per
 * SM sub-partition; their 128-byte pair records are most of its memory
 * traffic.  This walk tests the same tree's boxes in f32 (FMA, min/max) from
 * 64-byte records (FPair, zt_types.h) and keeps the primitive tests, the hit
 * records and all shading in f64, unchanged.
 *
 * Superset property.  A float box test here succeeds whenever the
 * reference's f64 test of the same box succeeds (same ray, same [tmin,
 * tmax]):
 *  - the ray is o + t d in f64; per axis the walk uses o32 = fl32(o),
 *    I = rcp(fl32(d)) (the hardware reciprocal, within 1 ulp, i.e. 2^-23
 *    relative; clamped to +-K, below) and n = fl32(-o32 I), and computes a
 *    plane distance as fl32(c I + off) with one FMA, c the float plane and
 *    off = n -+ w.  Against the exact (c - o) / d the error is at most
 *    2^-23 (2 |c| + 3.5 |o|) / |d| (rounding of d, of o, of the product n,
 *    of the FMA and of n -+ w, each at most 2^-24 relative, and the
 *    reciprocal's 2^-23);
 *  - the |c| part is covered by the records: every bound is moved outward by
 *    eps = 2^-20 M (M the largest |bound| on that axis; 4x the 2 2^-23 M
 *    needed), which moves a near plane's distance down and a far plane's up
 *    by eps / |d|;
 *  - the |o| part is covered per ray: w = 2^-20 |n| (2.3x the 3.5 2^-23 |o I|
 *    needed) is subtracted from near planes and added to far planes;
 *  - so each near distance is at most the exact one and each far distance at
 *    least the exact one, tmin is rounded down and tmax up, and an interval
 *    the exact test finds non-empty stays non-empty.  The f64 test's own
 *    rounding (2^-53 relative) is far inside these margins.
 *  - A zero or tiny direction component has its reciprocal clamped to +-K
 *    with K |o| <= 1e37 and K M <= 1e37 (M <= kFastMaxCoord), so no product
 *    overflows; the plane distances then keep their signs (the ray is inside
 *    or outside that slab), which is all the test uses on that axis.
 * Entry distances are lower bounds of the exact ones, so `entry.t > closest`
 * pruning against closest rounded up never drops a node the reference
 * visits, and leaves are tested with the reference's f64 primitive tests.
 * The closest hit found is therefore the least primitive distance over a
 * superset of the leaves the reference tests; it differs from the
 * reference's only where two primitives tie, or where the reference's own
 * f64 box test misses a primitive hit by rounding (a grazing ray).  Images
 * are held to a statistical bar (per-channel relative RMSE
 * and mean luminance against the oracle), not to bit equality.
 *
 * Stack entries are 8 bytes (packed payload word + float entry distance),
 * 4 bytes in the any-hit walk.
 */
#ifndef ZT_FAST_CUH
#define ZT_FAST_CUH

namespace zt {

/* Per-ray constants of the float slab test, as packed f32x2 operands: per
 * axis the reciprocal twice, and the offsets of the planes through a box's
 * lower and upper bound (the FPair layout's order). */
struct FRay {
  unsigned long long inv2[3];
  unsigned long long off2[3];
};

ZT_D unsigned long long f2_pack(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
/* Both plane distances of one axis: fl32(c * inv + off) for c = lower and
 * upper bound, each lane one FMA with a single rounding (as fmaf). */
ZT_D void f2_planes(unsigned long long box, unsigned long long inv2, unsigned long long off2, float& a, float& b) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(box), "l"(inv2), "l"(off2));
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(r));
}
/* Three-input minimum and maximum (sm_100). */
ZT_D float fmax3f(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}
ZT_D float fmin3f(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

/* Largest |origin| component the float test takes; rays from farther away
 * (a hit far out on an unbounded plane) use the f64 walk. */
constexpr float kFastMaxOrigin = 1e30f;

ZT_D bool fray_make(dv3 o, dv3 d, FRay& r) {
  const float o3[3] = {(float)o.x, (float)o.y, (float)o.z};
  const float d3[3] = {(float)d.x, (float)d.y, (float)d.z};
  const float om = fmaxf(fabsf(o3[0]), fmaxf(fabsf(o3[1]), fabsf(o3[2])));
  if (!(om <= kFastMaxOrigin)) return false;
  const float K = om > 1e7f ? 1e37f / om : 1e30f; /* K |o| <= 1e37, K * kFastMaxCoord <= 1e37 */
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float inv;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(d3[a])); /* within 1 ulp; +-0 (and flushed subnormals) give +-inf */
    if (!(fabsf(inv) <= K)) inv = copysignf(K, inv); /* +-inf (a zero component) and huge values */
    const float n = -o3[a] * inv;
    const float w = fabsf(n) * 0x1.0p-20f;
    /* lower plane nearer when inv >= 0: it takes n - w, the upper plane n + w */
    r.inv2[a] = f2_pack(inv, inv);
    r.off2[a] = inv >= 0.0f ? f2_pack(n - w, n + w) : f2_pack(n + w, n - w);
  }
  return true;
}

/* The f64 walks, outlined: the fast walks' fallback for far origins. */
__device__ __noinline__ int32_t scene_query_exact_outlined(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax,
                                                            double& t_out) {
  return scene_query_rt(sc, o, d, tmin, tmax, false, t_out);
}
__device__ __noinline__ bool scene_occluded_exact_outlined(const DevScene& sc, dv3 o, dv3 d, double tmin,
                                                           double tmax) {
  return scene_occluded(sc, o, d, tmin, tmax);
}

/* Float slab test of one box given as its three (lower, upper) axis pairs;
 * tnear is the (lower-bound) entry distance. */
ZT_D bool fslab(unsigned long long bx, unsigned long long by, unsigned long long bz, const FRay& r, float tmin,
                float tmax, float& tnear) {
  float a0, b0, a1, b1, a2, b2;
  f2_planes(bx, r.inv2[0], r.off2[0], a0, b0);
  f2_planes(by, r.inv2[1], r.off2[1], a1, b1);
  f2_planes(bz, r.inv2[2], r.off2[2], a2, b2);
  const float n = fmax3f(fminf(a0, b0), fminf(a1, b1), fmaxf(fminf(a2, b2), tmin));
  const float f = fmin3f(fmaxf(a0, b0), fmaxf(a1, b1), fminf(fmaxf(a2, b2), tmax));
  tnear = n;
  return n <= f;
}

/* One 64-byte record: both children's axis pairs and payload words. */
struct FRec {
  ulonglong2 q0, q1, q2;
  uint2 w;
};
ZT_D FRec frec_load(const FPair* p) {
  const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
  FRec r;
  r.q0 = __ldg(q);
  r.q1 = __ldg(q + 1);
  r.q2 = __ldg(q + 2);
  r.w = __ldg(reinterpret_cast<const uint2*>(q + 3));
  return r;
}
/* left x y = q0.x q0.y, left z = q1.x; right x = q1.y, right y z = q2.x q2.y */
ZT_D bool fslab_left(const FRec& r, const FRay& fr, float tmin, float tmax, float& t) {
  return fslab(r.q0.x, r.q0.y, r.q1.x, fr, tmin, tmax, t);
}
ZT_D bool fslab_right(const FRec& r, const FRay& fr, float tmin, float tmax, float& t) {
  return fslab(r.q1.y, r.q2.x, r.q2.y, fr, tmin, tmax, t);
}
ZT_D bool fslab_root(const DevScene& sc, const FRay& fr, float tmin, float tmax, float& t) {
  return fslab(f2_pack(sc.froot[0][0], sc.froot[0][1]), f2_pack(sc.froot[1][0], sc.froot[1][1]),
               f2_pack(sc.froot[2][0], sc.froot[2][1]), fr, tmin, tmax, t);
}

/* Scene.intersect (scene.zig:108-116) with the BVH walked over the float
 * records: nearest first by float entry distance (ties to the left child,
 * bvh.zig:111-116), pruning entries whose distance exceeds the closest hit,
 * f64 primitive tests; then the unbounded planes.  Return value and t_out as
 * scene_query_rt's (closest hit only). */
ZT_D int32_t scene_query_fast(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax, double& t_out) {
  double closest = tmax;
  int32_t best_k = -1;
  if (sc.has_root) {
    FRay fr;
    if (!fray_make(o, d, fr)) return scene_query_exact_outlined(sc, o, d, tmin, tmax, t_out);
    const float tmin32 = __double2float_rd(tmin);
    float cl32 = __double2float_ru(closest);
    float t;
    if (fslab_root(sc, fr, tmin32, cl32, t)) {
      uint2 stack[kStackSize]; /* (payload word, entry distance bits) */
      uint32_t w = sc.froot_word;
      float et = t;
      bool have = true;
      int sp = 0;
      for (;;) {
        if (!have) {
          if (sp == 0) break;
          const uint2 e = stack[--sp];
          w = e.x;
          et = __uint_as_float(e.y);
        }
        have = false;
        if (et > cl32) continue; /* bvh.zig:97, against closest rounded up */
        const uint32_t cnt = w >> kFastCountShift, first = w & kFastFirstMask;
        if (cnt > 0) {
          for (uint32_t k = first; k < first + cnt; ++k) {
            double th;
            if (bounded_t(sc.prims[k], o, d, tmin, closest, th)) {
              closest = th;
              best_k = (int32_t)k;
              cl32 = __double2float_ru(th);
            }
          }
          continue;
        }
        const FRec r = frec_load(sc.fpairs + first);
        float tl, tr;
        const bool hl = fslab_left(r, fr, tmin32, cl32, tl);
        const bool hr = fslab_right(r, fr, tmin32, cl32, tr);
        if (hl && hr) { /* push the farther child; the nearer one is next */
          const bool near_left = tl <= tr;
          stack[sp] = make_uint2(near_left ? r.w.y : r.w.x, __float_as_uint(near_left ? tr : tl));
          sp += 1;
          w = near_left ? r.w.x : r.w.y;
          et = near_left ? tl : tr;
          have = true;
        } else if (hl || hr) {
          w = hl ? r.w.x : r.w.y;
          et = hl ? tl : tr;
          have = true;
        }
      }
    }
  }
  for (uint32_t i = 0; i < sc.n_planes; ++i) { /* geometry.zig:129-139 */
    double th;
    if (plane_prim_t(sc.planes[i], o, d, tmin, closest, th)) {
      closest = th;
      best_k = -2 - (int32_t)i;
    }
  }
  t_out = closest;
  return best_k;
}

/* Shadow query over the float records: whether any primitive is hit in
 * (tmin, tmax).  The leaves it tests are a superset of the leaves the f64
 * walk tests, and any primitive hit below tmax is an occluder whichever walk
 * finds it.  Farther child first, as scene_occluded. */
ZT_D bool scene_occluded_fast(const DevScene& sc, dv3 o, dv3 d, double tmin, double tmax) {
  if (sc.has_root) {
    FRay fr;
    if (!fray_make(o, d, fr)) return scene_occluded_exact_outlined(sc, o, d, tmin, tmax);
    const float tmin32 = __double2float_rd(tmin), tmax32 = __double2float_ru(tmax);
    float t;
    if (fslab_root(sc, fr, tmin32, tmax32, t)) {
      uint32_t stack[kStackSize];
      uint32_t w = sc.froot_word;
      bool have = true;
      int sp = 0;
      for (;;) {
        if (!have) {
          if (sp == 0) break;
          w = stack[--sp];
        }
        have = false;
        const uint32_t cnt = w >> kFastCountShift, first = w & kFastFirstMask;
        if (cnt > 0) {
          for (uint32_t k = first; k < first + cnt; ++k) {
            double th;
            if (prim_t(sc.prims[k], o, d, tmin, tmax, th)) return true;
          }
          continue;
        }
        const FRec r = frec_load(sc.fpairs + first);
        float tl, tr;
        const bool hl = fslab_left(r, fr, tmin32, tmax32, tl);
        const bool hr = fslab_right(r, fr, tmin32, tmax32, tr);
        if (hl && hr) {
          const bool left_first = tl > tr; /* the farther child first */
          stack[sp++] = left_first ? r.w.y : r.w.x;
          w = left_first ? r.w.x : r.w.y;
          have = true;
        } else if (hl || hr) {
          w = hl ? r.w.x : r.w.y;
          have = true;
        }
      }
    }
  }
  for (uint32_t i = 0; i < sc.n_planes; ++i) {
    double th;
    if (prim_t(sc.planes[i], o, d, tmin, tmax, th)) return true;
  }
  return false;
}

}  // namespace zt

#endif

/*
 * zt_types.h -- device-resident scene layout (shared by the host builder and
 * the CUDA kernels).
 *
 * The reference keeps a flat `[]Node` of 56-byte nodes whose two children are
 * adjacent (src/bvh.zig:22-33) and a `[]Shape` tagged union indexed through a
 * permutation `indices` (src/bvh.zig:35-38).  The device layout regroups the
 * same data for one-line-per-visit access without changing any value:
 *
 *  - DPair: the two children of one interior node, both boxes plus each
 *    child's payload, in one 128-byte record (one L2 line).  A traversal step
 *    that pops an interior node reads exactly one record, where the reference
 *    reads nodes[l] and nodes[l+1].  Record r holds reference nodes 2r+1 and
 *    2r+2 (left children are always odd: the node array grows in pairs).
 *  - Payload of a child: a leaf stores (first, count>0) into the reordered
 *    primitive array; an interior child stores (record of its children, 0).
 *  - DPrim: bounded shapes reordered into BVH leaf order (prims[k] =
 *    shapes[indices[k]]), so a leaf's primitives are contiguous.  Triangles
 *    store v0, e1 = v1 - v0, e2 = v2 - v0 (the same subtractions the
 *    reference repeats per test, src/geometry.zig:84-85, done once on the
 *    host with identical rounding).
 */
#ifndef ZT_TYPES_H
#define ZT_TYPES_H

#include <stdint.h>

#if defined(__CUDACC__)
#define ZT_ALIGN(n) __align__(n)
#else
#define ZT_ALIGN(n) alignas(n)
#endif

namespace zt {

enum PrimKind : uint32_t { kSphere = 0, kTriangle = 1, kPlane = 2 };
enum MatKind : uint32_t { kLambertian = 0, kMetal = 1, kDielectric = 2, kEmissive = 3 };

/* 80 bytes. sphere: a[0..2] center, a[3] radius.  triangle: a[0..2] v0,
 * a[3..5] e1, a[6..8] e2.  plane: a[0..2] point, a[3..5] normal. */
struct ZT_ALIGN(16) DPrim {
  double a[9];
  uint32_t material;
  uint32_t kind;
};

/* 128 bytes: children c = 0, 1 of one interior node. */
struct ZT_ALIGN(128) DPair {
  double lo[2][3];
  double hi[2][3];
  uint32_t first[2];
  uint32_t count[2];
};

/* 64 bytes: the same two children as a DPair, for the fast traversal
 * (zt_fast.cuh).  Boxes are single precision and conservative: every bound
 * is moved outward by eps[axis] = 2^-20 * max(|root lo|, |root hi|) on that
 * axis and then rounded outward to float, so the box contains the f64 box
 * with a margin that covers the float slab test's rounding.  Each axis of a
 * child is a (lower, upper) pair in adjacent words, the operand layout of one
 * packed f32x2 FMA that gives both plane distances.  word[c] packs the
 * child's payload: count << 28 | first (count 0: first is the record of the
 * child's own children). */
struct ZT_ALIGN(64) FPair {
  float b[2][3][2]; /* [child][axis][lower, upper] */
  uint32_t word[2];
  uint32_t pad[2];
};
constexpr uint32_t kFastCountShift = 28;
constexpr uint32_t kFastFirstMask = (1u << kFastCountShift) - 1;
constexpr uint32_t kFastMaxLeaf = (1u << (32 - kFastCountShift)) - 1;
/* Largest |coordinate| (of the scene's bounds and of ray origins) the float
 * slab test handles: products with the clamped reciprocal stay finite. */
constexpr double kFastMaxCoord = 1e7;

struct ZT_ALIGN(16) DMat {
  double color[3];
  double param;
  uint32_t kind;
  uint32_t pad[3];
};

/* Light (src/light.zig:30-35) with the per-light constants the reference
 * recomputes on every call precomputed on the host with identical rounding:
 * area = triangleArea (light.zig:42-44) and the unit normal of
 * (v1 - v0) x (v2 - v0) (light.zig:133). */
struct ZT_ALIGN(16) DLight {
  double v[9];       /* triangle v0, v1, v2; sphere center.xyz, radius */
  double radiance[3];
  double weight;
  double area;       /* triangle only */
  double normal[3];  /* triangle only */
  uint32_t kind;
  uint32_t material; /* the emitter's material (differentiable form) */
};

struct DCamera {
  double origin[3], upper_left[3], horizontal[3], vertical[3], u[3], v[3];
  double lens_radius;
};

struct DBackground {
  double a[3], b[3];
  uint32_t kind;
  uint32_t pad;
};

/* Everything a kernel needs, passed by value. */
struct DevScene {
  const DPrim* prims;
  const int32_t* prim_ids;  /* original bounded-shape index of prims[k] */
  const DPair* pairs;
  const DPrim* planes;
  const DMat* mats;
  const DLight* lights;
  const double* cdf;
  double root_lo[3], root_hi[3];
  uint32_t root_first, root_count;
  uint32_t has_root;  /* 0 when there are no bounded shapes */
  uint32_t n_prims, n_planes, n_mats, n_lights;
  uint32_t pad;
  double total;       /* Lights.total */
  DBackground bg;
  /* fast traversal (zt_fast.cuh): conservative float records and root box */
  const FPair* fpairs;
  float froot[3][2]; /* root box, [axis][lower, upper] as in FPair */
  uint32_t froot_word;
  uint32_t fast_ok;   /* 1 when the fast records exist (leaves <= 15 primitives, bounds within kFastMaxCoord) */
};

struct RenderParams {
  DCamera cam;
  uint64_t width, height, spp, max_depth, seed;
  uint64_t row0, rows; /* the band of image rows rendered; output row 0 is image row row0 */
  uint32_t use_nee;  /* light_sampling && !lights.isEmpty() */
  uint32_t pad;
};

}  // namespace zt

#endif

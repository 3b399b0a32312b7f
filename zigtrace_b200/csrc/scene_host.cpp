/*
 * scene_host.cpp -- Scene construction, BVH build, emitter table and camera
 * set-up on the host (the part of the reference that runs before the timed
 * render: src/scene.zig:53-96, src/bvh.zig:41-262, src/light.zig:68-94,
 * src/camera.zig:29-55), and the C-ABI entry points that expose them.
 *
 * Compiled with -ffp-contract=off: the node bounds, SAH costs, light weights
 * and camera vectors round exactly as the reference's strict-float code, so
 * the uploaded BVH is the reference's BVH node for node.
 */
#include "scene_host.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <new>

namespace zt {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

zt_status fail(zt_status code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

/* ------------------------------------------------------------ AABB ---- */
/* src/aabb.zig */
struct Box {
  double mn[3], mx[3];
};

static inline Box box_empty() {
  Box b;
  for (int a = 0; a < 3; ++a) { b.mn[a] = INFINITY; b.mx[a] = -INFINITY; }
  return b;
}
static inline void box_merge(Box& a, const Box& b) { /* aabb.zig:21-23 */
  for (int k = 0; k < 3; ++k) { a.mn[k] = fmin(a.mn[k], b.mn[k]); a.mx[k] = fmax(a.mx[k], b.mx[k]); }
}
static inline void box_include(Box& a, const double p[3]) { /* aabb.zig:25-27 */
  for (int k = 0; k < 3; ++k) { a.mn[k] = fmin(a.mn[k], p[k]); a.mx[k] = fmax(a.mx[k], p[k]); }
}
static inline bool box_is_empty(const Box& a) {
  return a.mn[0] > a.mx[0] || a.mn[1] > a.mx[1] || a.mn[2] > a.mx[2];
}
static inline double box_area(const Box& a) { /* aabb.zig:53-57 */
  if (box_is_empty(a)) return 0;
  const double ex = a.mx[0] - a.mn[0], ey = a.mx[1] - a.mn[1], ez = a.mx[2] - a.mn[2];
  return 2.0 * (ex * ey + ey * ez + ez * ex);
}
static inline int box_longest_axis(const Box& a) { /* aabb.zig:59-63 */
  const double ex = a.mx[0] - a.mn[0], ey = a.mx[1] - a.mn[1], ez = a.mx[2] - a.mn[2];
  if (ex >= ey && ex >= ez) return 0;
  return ey >= ez ? 1 : 2;
}

/* Shape.bounds, geometry.zig:54-57, 101-103; returns false for planes. */
static bool shape_bounds(const zt_shape& s, Box& b) {
  if (s.kind == ZT_SPHERE) {
    const double r = fabs(s.p[3]);
    for (int k = 0; k < 3; ++k) { b.mn[k] = s.p[k] - r; b.mx[k] = s.p[k] + r; }
    return true;
  }
  if (s.kind == ZT_TRIANGLE) {
    for (int k = 0; k < 3; ++k) { b.mn[k] = fmin(s.p[k], s.p[3 + k]); b.mx[k] = fmax(s.p[k], s.p[3 + k]); }
    box_include(b, s.p + 6);
    const double delta = 1e-6; /* Aabb.pad, aabb.zig:30-39 */
    for (int k = 0; k < 3; ++k)
      if (b.mx[k] - b.mn[k] < delta) { b.mn[k] -= delta / 2; b.mx[k] += delta / 2; }
    return true;
  }
  return false;
}

/* ------------------------------------------------------------- BVH ---- */
/* src/bvh.zig:16-262 */
constexpr int kBinCount = 12;
constexpr uint32_t kMaxLeafSize = 4;
constexpr size_t kMaxDepth = 64;
constexpr double kTraversalCost = 1.0;

struct Builder {
  std::vector<HostNode>& nodes;
  uint32_t* indices;
  const std::vector<Box>& boxes;
  const std::vector<double>& cent;  /* 3 per primitive */

  static size_t bin_of(double c, double lo, double extent) { /* bvh.zig:258-262 */
    const double f = (c - lo) / extent * (double)kBinCount;
    return (size_t)fmax(0.0, fmin(f, (double)(kBinCount - 1)));
  }

  struct Split { int axis; size_t bin; double cost; bool valid; };

  Split find_split(const uint32_t* range, uint32_t count, const Box& bounds, const Box& cb) const {
    /* bvh.zig:211-256 */
    Split best{0, 0, 0.0, false};
    const double parent_area = box_area(bounds);
    if (parent_area <= 0) return best;
    for (int axis = 0; axis < 3; ++axis) {
      const double lo = cb.mn[axis];
      const double extent = cb.mx[axis] - lo;
      if (!(extent > 0)) continue;
      Box bin_box[kBinCount];
      size_t bin_n[kBinCount];
      for (int i = 0; i < kBinCount; ++i) { bin_box[i] = box_empty(); bin_n[i] = 0; }
      for (uint32_t j = 0; j < count; ++j) {
        const uint32_t idx = range[j];
        const size_t b = bin_of(cent[3 * (size_t)idx + axis], lo, extent);
        bin_n[b] += 1;
        box_merge(bin_box[b], boxes[idx]);
      }
      double right_area[kBinCount];
      size_t right_n[kBinCount];
      Box acc = box_empty();
      size_t acc_n = 0;
      for (int i = kBinCount - 1; i >= 0; --i) {
        box_merge(acc, bin_box[i]);
        acc_n += bin_n[i];
        right_area[i] = box_area(acc);
        right_n[i] = acc_n;
      }
      acc = box_empty();
      acc_n = 0;
      for (int b = 0; b < kBinCount - 1; ++b) {
        box_merge(acc, bin_box[b]);
        acc_n += bin_n[b];
        const size_t rn = right_n[b + 1];
        if (acc_n == 0 || rn == 0) continue;
        const double cost =
            kTraversalCost + (box_area(acc) * (double)acc_n + right_area[b + 1] * (double)rn) / parent_area;
        if (!best.valid || cost < best.cost) best = Split{axis, (size_t)b, cost, true};
      }
    }
    return best;
  }

  void make_children(size_t node_idx, uint32_t first, uint32_t left_count, uint32_t count, size_t level) {
    /* bvh.zig:187-195 */
    const uint32_t left = (uint32_t)nodes.size();
    HostNode e;
    for (int k = 0; k < 3; ++k) { e.bmin[k] = INFINITY; e.bmax[k] = -INFINITY; }
    e.first = first;
    e.count = left_count;
    nodes.push_back(e);
    e.first = first + left_count;
    e.count = count - left_count;
    nodes.push_back(e);
    nodes[node_idx].first = left;
    nodes[node_idx].count = 0;
    subdivide(left, level + 1);
    subdivide(left + 1, level + 1);
  }

  void subdivide(size_t node_idx, size_t level) { /* bvh.zig:148-185 */
    const uint32_t first = nodes[node_idx].first;
    const uint32_t count = nodes[node_idx].count;
    uint32_t* range = indices + first;
    Box bounds = box_empty(), cb = box_empty();
    for (uint32_t j = 0; j < count; ++j) {
      const uint32_t i = range[j];
      box_merge(bounds, boxes[i]);
      box_include(cb, &cent[3 * (size_t)i]);
    }
    for (int k = 0; k < 3; ++k) { nodes[node_idx].bmin[k] = bounds.mn[k]; nodes[node_idx].bmax[k] = bounds.mx[k]; }
    if (count <= 1 || level >= kMaxDepth) return;
    const double leaf_cost = (double)count;
    const Split split = find_split(range, count, bounds, cb);
    if (!split.valid) {
      if (count <= kMaxLeafSize) return;
      /* splitMedian, bvh.zig:197-209: std.mem.sort is stable */
      const int axis = box_longest_axis(cb);
      std::stable_sort(range, range + count, [&](uint32_t a, uint32_t b) {
        return cent[3 * (size_t)a + axis] < cent[3 * (size_t)b + axis];
      });
      make_children(node_idx, first, count / 2, count, level);
      return;
    }
    if (count <= kMaxLeafSize && split.cost >= leaf_cost) return;
    const int axis = split.axis;
    const double lo = cb.mn[axis];
    const double extent = cb.mx[axis] - lo;
    uint32_t mid = 0;
    for (uint32_t j = 0; j < count; ++j) {
      if (bin_of(cent[3 * (size_t)range[j] + axis], lo, extent) <= split.bin) {
        std::swap(range[mid], range[j]);
        mid += 1;
      }
    }
    make_children(node_idx, first, mid, count, level);
  }
};

static zt_status build_bvh(zt_scene* s) { /* Bvh.build, bvh.zig:41-67 */
  const size_t n = s->shapes.size();
  s->nodes.clear();
  s->indices.clear();
  if (n == 0) return ZT_OK;
  if (n > 0xFFFFFFFFull / 2) return fail(ZT_ERR_TOO_MANY_PRIMITIVES, "TooManyPrimitives: more than 2^31 bounded shapes");
  std::vector<Box> boxes(n);
  std::vector<double> cent(3 * n);
  s->indices.resize(n);
  for (size_t i = 0; i < n; ++i) {
    s->indices[i] = (uint32_t)i;
    if (!shape_bounds(s->shapes[i], boxes[i])) return fail(ZT_ERR_UNBOUNDED_SHAPE, "UnboundedShape");
    for (int k = 0; k < 3; ++k) cent[3 * i + k] = (boxes[i].mn[k] + boxes[i].mx[k]) * 0.5; /* centroid */
  }
  s->nodes.reserve(2 * n - 1);
  HostNode root;
  for (int k = 0; k < 3; ++k) { root.bmin[k] = INFINITY; root.bmax[k] = -INFINITY; }
  root.first = 0;
  root.count = (uint32_t)n;
  s->nodes.push_back(root);
  Builder b{s->nodes, s->indices.data(), boxes, cent};
  b.subdivide(0, 0);
  return ZT_OK;
}

/* ---------------------------------------------------------- Lights ---- */
/* src/light.zig:68-94 */
static inline double tri_area(const double* p) { /* light.zig:42-44 */
  const double e1[3] = {p[3] - p[0], p[4] - p[1], p[5] - p[2]};
  const double e2[3] = {p[6] - p[0], p[7] - p[1], p[8] - p[2]};
  const double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  return 0.5 * sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
}

static const double kPi = 3.14159265358979323846;

static zt_status build_lights(zt_scene* s) {
  s->lights.clear();
  s->cdf.clear();
  for (const zt_shape& sh : s->shapes) {
    double area;
    if (sh.kind == ZT_TRIANGLE) area = tri_area(sh.p);
    else if (sh.kind == ZT_SPHERE) area = sh.p[3] > 0 ? 4 * kPi * sh.p[3] * sh.p[3] : 0;
    else continue;
    const zt_material& m = s->materials[sh.material];
    if (m.kind != ZT_EMISSIVE) continue;
    const double lum = 0.2126 * m.color.x + 0.7152 * m.color.y + 0.0722 * m.color.z;
    const double weight = lum * area;
    if (!(weight > 0) || !isfinite(weight)) continue;
    HostLight L;
    L.shape = sh;
    L.radiance[0] = m.color.x;
    L.radiance[1] = m.color.y;
    L.radiance[2] = m.color.z;
    L.weight = weight;
    s->lights.push_back(L);
  }
  double sum = 0;
  for (const HostLight& L : s->lights) {
    sum += L.weight;
    s->cdf.push_back(sum);
  }
  s->total = sum;
  return ZT_OK;
}

zt_status build_scene(zt_scene* s, bool device, bool* used_device, double* build_ms) { /* Scene.build, scene.zig:92-96 */
  for (const zt_shape& sh : s->shapes)
    if (sh.material >= s->materials.size()) return fail(ZT_ERR_INVALID_ARGUMENT, "shape refers to an undefined material");
  for (const zt_shape& sh : s->planes)
    if (sh.material >= s->materials.size()) return fail(ZT_ERR_INVALID_ARGUMENT, "plane refers to an undefined material");
  release_staging(s);
  s->built = false;
  s->pilot_valid = false;
  zt_status rc;
  if (used_device) *used_device = false;
  try {
    rc = ZT_DEVICE_BUILD_FALLBACK;
    if (device) {
      rc = device_build_bvh(s, build_ms);
      if (rc == ZT_OK && used_device) *used_device = true;
    }
    if (rc == ZT_DEVICE_BUILD_FALLBACK) rc = build_bvh(s);
    if (rc == ZT_OK) rc = build_lights(s);
  } catch (const std::bad_alloc&) {
    return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory during Scene.build");
  }
  if (rc == ZT_OK) s->built = true;
  return rc;
}

/* Scene.build with a BVH built elsewhere (the reference's own Bvh.build,
 * bvh.zig:41-67, for a caller that already holds it): the tree is checked
 * to be one this renderer can traverse exactly as the reference does, then
 * used as given; the emitter table is built as Scene.build builds it
 * (light.zig:68-94).  The checks: indices is a permutation of the bounded
 * shapes; node 0 is the root; an interior node's children sit at first and
 * first + 1 with first odd (the reference appends children in pairs after
 * the root, so every pair of siblings starts at an odd index); every node
 * but the root is the child of exactly one node; no node is deeper than
 * the reference's max_depth (64), so the traversal stack of max_depth + 2
 * entries (bvh.zig:87) cannot overflow; leaves cover [0, n) exactly once. */
zt_status import_bvh(zt_scene* s, const zt_bvh_node* nodes, size_t n_nodes, const uint32_t* indices, size_t n_idx) {
  for (const zt_shape& sh : s->shapes)
    if (sh.material >= s->materials.size()) return fail(ZT_ERR_INVALID_ARGUMENT, "shape refers to an undefined material");
  for (const zt_shape& sh : s->planes)
    if (sh.material >= s->materials.size()) return fail(ZT_ERR_INVALID_ARGUMENT, "plane refers to an undefined material");
  const size_t n = s->shapes.size();
  auto bad = [](const std::string& why) { return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_set_bvh: " + why); };
  if (n > 0xFFFFFFFFull / 2) return fail(ZT_ERR_TOO_MANY_PRIMITIVES, "TooManyPrimitives"); /* bvh.zig:44 */
  if (n_idx != n) return bad("indices must hold one entry per bounded shape");
  if (n == 0) {
    if (n_nodes != 0) return bad("a scene without bounded shapes has no nodes");
  } else {
    if (!nodes || !indices) return bad("NULL nodes or indices");
    if (n_nodes == 0 || n_nodes > 2 * n - 1 || n_nodes % 2 == 0)
      return bad("node count must be odd and between 1 and 2n-1");
  }
  std::vector<uint8_t> seen(n, 0);
  for (size_t i = 0; i < n; ++i) {
    if (indices[i] >= n || seen[indices[i]]) return bad("indices is not a permutation of the bounded shapes");
    seen[indices[i]] = 1;
  }
  std::vector<uint8_t> level(n_nodes, 0), reached(n_nodes, 0);
  std::vector<uint8_t> covered(n, 0);
  if (n_nodes) reached[0] = 1;
  /* children always follow their parent (first is odd and > parent), so one
   * pass in index order visits every parent before its children */
  for (size_t i = 0; i < n_nodes; ++i) {
    if (!reached[i]) return bad("node " + std::to_string(i) + " is not reachable from the root");
    const zt_bvh_node& nd = nodes[i];
    if (nd.count == 0) {
      const uint64_t l = nd.first;
      if (l % 2 == 0 || l <= i || l + 1 >= n_nodes)
        return bad("interior node " + std::to_string(i) + " has children outside the node array or not in a pair");
      if (level[i] >= kMaxDepth) return bad("tree deeper than 64 levels");
      for (uint64_t c = l; c <= l + 1; ++c) {
        if (reached[c]) return bad("node " + std::to_string(c) + " has two parents");
        reached[c] = 1;
        level[c] = level[i] + 1;
      }
    } else {
      if ((uint64_t)nd.first + nd.count > n) return bad("leaf " + std::to_string(i) + " reaches past the last shape");
      for (uint64_t k = nd.first; k < (uint64_t)nd.first + nd.count; ++k) {
        if (covered[k]) return bad("two leaves share shape position " + std::to_string(k));
        covered[k] = 1;
      }
    }
  }
  for (size_t k = 0; k < n; ++k)
    if (!covered[k]) return bad("shape position " + std::to_string(k) + " is in no leaf");
  release_staging(s);
  s->built = false;
  s->pilot_valid = false;
  try {
    s->nodes.resize(n_nodes);
    for (size_t i = 0; i < n_nodes; ++i) {
      HostNode& h = s->nodes[i];
      h.bmin[0] = nodes[i].bmin.x; h.bmin[1] = nodes[i].bmin.y; h.bmin[2] = nodes[i].bmin.z;
      h.bmax[0] = nodes[i].bmax.x; h.bmax[1] = nodes[i].bmax.y; h.bmax[2] = nodes[i].bmax.z;
      h.first = nodes[i].first;
      h.count = nodes[i].count;
    }
    s->indices.assign(indices, indices + n);
    const zt_status rc = build_lights(s);
    if (rc != ZT_OK) return rc;
  } catch (const std::bad_alloc&) {
    return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory in zt_scene_set_bvh");
  }
  s->built = true;
  return ZT_OK;
}

/* ---------------------------------------------------------- Camera ---- */
static inline void v3_sub(const zt_vec3& a, const zt_vec3& b, double o[3]) {
  o[0] = a.x - b.x; o[1] = a.y - b.y; o[2] = a.z - b.z;
}
static inline void v3_cross(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double v3_len(const double a[3]) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }
static inline void v3_normalize(double a[3]) { /* Vec3.normalize = scale(1/len) */
  const double inv = 1.0 / v3_len(a);
  a[0] = a[0] * inv; a[1] = a[1] * inv; a[2] = a[2] * inv;
}

DCamera camera_init(const zt_camera_config& cfg, double aspect) { /* camera.zig:29-55 */
  DCamera c;
  const double theta = cfg.vfov * (kPi / 180.0); /* std.math.degreesToRadians */
  const double half_h = tan(theta / 2);
  const double viewport_h = 2.0 * half_h;
  const double viewport_w = aspect * viewport_h;
  double w[3], u[3], v[3], upv[3] = {cfg.up.x, cfg.up.y, cfg.up.z};
  v3_sub(cfg.look_from, cfg.look_at, w);
  v3_normalize(w);
  v3_cross(upv, w, u);
  v3_normalize(u);
  v3_cross(w, u, v);
  double view[3];
  v3_sub(cfg.look_from, cfg.look_at, view);
  const double focus = cfg.has_focus_dist ? cfg.focus_dist : v3_len(view);
  const double hs = viewport_w * focus, vs = -viewport_h * focus;
  const double from[3] = {cfg.look_from.x, cfg.look_from.y, cfg.look_from.z};
  for (int k = 0; k < 3; ++k) {
    c.horizontal[k] = u[k] * hs;
    c.vertical[k] = v[k] * vs;
  }
  for (int k = 0; k < 3; ++k) {
    /* look_from.sub(w.scale(focus)).sub(horizontal.scale(0.5)).sub(vertical.scale(0.5)) */
    c.upper_left[k] = ((from[k] - w[k] * focus) - c.horizontal[k] * 0.5) - c.vertical[k] * 0.5;
    c.origin[k] = from[k];
    c.u[k] = u[k];
    c.v[k] = v[k];
  }
  c.lens_radius = cfg.aperture / 2;
  return c;
}

/* ---------------------------------------------------------- Flatten ---- */
static DPrim to_prim(const zt_shape& s) {
  DPrim p;
  memset(&p, 0, sizeof p);
  p.material = s.material;
  p.kind = s.kind;
  if (s.kind == ZT_TRIANGLE) {
    for (int k = 0; k < 3; ++k) {
      p.a[k] = s.p[k];
      p.a[3 + k] = s.p[3 + k] - s.p[k]; /* e1 = v1 - v0 */
      p.a[6 + k] = s.p[6 + k] - s.p[k]; /* e2 = v2 - v0 */
    }
  } else {
    for (int k = 0; k < 9; ++k) p.a[k] = s.p[k];
  }
  return p;
}

/* Nearest float at or below / at or above x. */
static float f32_down(double x) {
  float f = (float)x;
  if ((double)f > x) f = std::nextafterf(f, -INFINITY);
  return f;
}
static float f32_up(double x) {
  float f = (float)x;
  if ((double)f < x) f = std::nextafterf(f, INFINITY);
  return f;
}

/* The fast traversal's float records (zt_types.h FPair): every box of the
 * f64 tree moved outward by eps[axis] = 2^-20 * M[axis], M the largest
 * |bound| of the root box on that axis, then rounded outward.  The margin
 * covers the float slab test's rounding of box coordinates (the error
 * analysis is in zt_fast.cuh), so a ray whose f64 slab test reaches a box
 * also reaches its float copy.  Left empty (fast traversal unavailable) when
 * a leaf holds more than kFastMaxLeaf primitives, the tree is too large for
 * the packed payload word, or the bounds exceed kFastMaxCoord. */
static void make_fast_records(const zt_scene* s, FlatScene* f) {
  DevScene& v = f->view;
  v.fast_ok = 0;
  f->fpairs.clear();
  const size_t nn = s->nodes.size();
  if (nn == 0 || s->shapes.size() > kFastFirstMask || f->pairs.size() > kFastFirstMask) return;
  double eps[3];
  for (int k = 0; k < 3; ++k) {
    const double m = std::max(std::fabs(s->nodes[0].bmin[k]), std::fabs(s->nodes[0].bmax[k]));
    if (!(m <= kFastMaxCoord)) return; /* also rejects NaN */
    eps[k] = std::ldexp(m, -20);
  }
  for (const HostNode& nd : s->nodes)
    if (nd.count > kFastMaxLeaf) return;
  auto word = [&](uint32_t c) -> uint32_t {
    const HostNode& nd = s->nodes[c];
    return nd.count > 0 ? (nd.count << kFastCountShift) | nd.first : (nd.first - 1) / 2;
  };
  f->fpairs.assign(f->pairs.size(), FPair{});
  for (size_t i = 0; i < nn; ++i) {
    const HostNode& nd = s->nodes[i];
    if (nd.count > 0) continue;
    FPair& pr = f->fpairs[(nd.first - 1) / 2];
    for (int c = 0; c < 2; ++c) {
      const HostNode& ch = s->nodes[nd.first + c];
      for (int k = 0; k < 3; ++k) {
        pr.b[c][k][0] = f32_down(ch.bmin[k] - eps[k]);
        pr.b[c][k][1] = f32_up(ch.bmax[k] + eps[k]);
      }
      pr.word[c] = word(nd.first + c);
    }
  }
  for (int k = 0; k < 3; ++k) {
    v.froot[k][0] = f32_down(s->nodes[0].bmin[k] - eps[k]);
    v.froot[k][1] = f32_up(s->nodes[0].bmax[k] + eps[k]);
  }
  v.froot_word = word(0);
  v.fast_ok = 1;
}

void flatten_scene(const zt_scene* s, FlatScene* f) {
  const size_t n = s->shapes.size();
  f->prims.resize(n);
  f->prim_ids.resize(n);
  for (size_t k = 0; k < n; ++k) {
    f->prims[k] = to_prim(s->shapes[s->indices[k]]);
    f->prim_ids[k] = (int32_t)s->indices[k];
  }
  DevScene& v = f->view;
  memset(&v, 0, sizeof v);
  const size_t nn = s->nodes.size();
  f->pairs.assign(nn > 1 ? (nn - 1) / 2 : 0, DPair{});
  auto payload = [&](uint32_t c, uint32_t& first, uint32_t& count) {
    const HostNode& nd = s->nodes[c];
    if (nd.count > 0) { first = nd.first; count = nd.count; }
    else { first = (nd.first - 1) / 2; count = 0; }
  };
  for (size_t i = 0; i < nn; ++i) {
    const HostNode& nd = s->nodes[i];
    if (nd.count > 0) continue;
    DPair& pr = f->pairs[(nd.first - 1) / 2];
    for (int c = 0; c < 2; ++c) {
      const HostNode& ch = s->nodes[nd.first + c];
      for (int k = 0; k < 3; ++k) { pr.lo[c][k] = ch.bmin[k]; pr.hi[c][k] = ch.bmax[k]; }
      payload(nd.first + c, pr.first[c], pr.count[c]);
    }
  }
  if (nn > 0) {
    v.has_root = 1;
    for (int k = 0; k < 3; ++k) { v.root_lo[k] = s->nodes[0].bmin[k]; v.root_hi[k] = s->nodes[0].bmax[k]; }
    payload(0, v.root_first, v.root_count);
  }
  make_fast_records(s, f);
  f->planes.resize(s->planes.size());
  for (size_t i = 0; i < s->planes.size(); ++i) f->planes[i] = to_prim(s->planes[i]);
  f->mats.resize(s->materials.size());
  for (size_t i = 0; i < s->materials.size(); ++i) {
    DMat& m = f->mats[i];
    memset(&m, 0, sizeof m);
    m.color[0] = s->materials[i].color.x;
    m.color[1] = s->materials[i].color.y;
    m.color[2] = s->materials[i].color.z;
    m.param = s->materials[i].param;
    m.kind = s->materials[i].kind;
  }
  f->lights.resize(s->lights.size());
  for (size_t i = 0; i < s->lights.size(); ++i) {
    const HostLight& L = s->lights[i];
    DLight& d = f->lights[i];
    memset(&d, 0, sizeof d);
    d.kind = L.shape.kind;
    for (int k = 0; k < 9; ++k) d.v[k] = L.shape.p[k];
    for (int k = 0; k < 3; ++k) d.radiance[k] = L.radiance[k];
    d.weight = L.weight;
    d.material = L.shape.material;
    if (L.shape.kind == ZT_TRIANGLE) {
      d.area = tri_area(L.shape.p);
      double e1[3], e2[3], nrm[3];
      for (int k = 0; k < 3; ++k) { e1[k] = L.shape.p[3 + k] - L.shape.p[k]; e2[k] = L.shape.p[6 + k] - L.shape.p[k]; }
      v3_cross(e1, e2, nrm);
      v3_normalize(nrm);
      for (int k = 0; k < 3; ++k) d.normal[k] = nrm[k];
    }
  }
  f->cdf = s->cdf;
  v.n_prims = (uint32_t)n;
  v.n_planes = (uint32_t)s->planes.size();
  v.n_mats = (uint32_t)s->materials.size();
  v.n_lights = (uint32_t)s->lights.size();
  v.total = s->total;
  const zt_background& bg = s->background;
  v.bg.kind = bg.kind;
  v.bg.a[0] = bg.a.x; v.bg.a[1] = bg.a.y; v.bg.a[2] = bg.a.z;
  v.bg.b[0] = bg.b.x; v.bg.b[1] = bg.b.y; v.bg.b[2] = bg.b.z;
}

static size_t depth_from(const zt_scene* s, uint32_t i) { /* bvh.zig:128-137 */
  const HostNode& n = s->nodes[i];
  if (n.count > 0) return 1;
  return 1 + std::max(depth_from(s, n.first), depth_from(s, n.first + 1));
}

}  // namespace zt

using namespace zt;

/* --------------------------------------------------------------- C ABI ---- */
extern "C" {

zt_status zt_scene_create(zt_scene** out) { /* Scene.init, scene.zig:53-55 */
  if (!out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_create: out is NULL");
  zt_scene* s = new (std::nothrow) zt_scene();
  if (!s) return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory");
  s->camera = zt_camera_config{{0, 0, 0}, {0, 0, -1}, {0, 1, 0}, 60.0, 0.0, 0.0, 0u, 0u};
  s->background = zt_background{ZT_BG_SKY, 0u, {1, 1, 1}, {0.5, 0.7, 1.0}};
  *out = s;
  return ZT_OK;
}

void zt_scene_destroy(zt_scene* s) {
  if (!s) return;
  release_staging(s);
  delete s;
}

zt_status zt_scene_add_material(zt_scene* s, const zt_material* m, uint32_t* id_out) {
  if (!s || !m) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_add_material: NULL argument");
  if (m->kind > ZT_EMISSIVE) return fail(ZT_ERR_INVALID_ARGUMENT, "unknown material kind");
  release_staging(s);
  s->built = false;
  s->materials.push_back(*m);
  if (id_out) *id_out = (uint32_t)(s->materials.size() - 1);
  return ZT_OK;
}

zt_status zt_scene_add_materials(zt_scene* s, const zt_material* m, size_t n, uint32_t* first_id_out) {
  if (!s || (!m && n)) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_add_materials: NULL argument");
  for (size_t i = 0; i < n; ++i)
    if (m[i].kind > ZT_EMISSIVE) return fail(ZT_ERR_INVALID_ARGUMENT, "unknown material kind");
  if (s->materials.size() + n > 0xFFFFFFFFull) return fail(ZT_ERR_INVALID_ARGUMENT, "too many materials");
  release_staging(s);
  s->built = false;
  if (first_id_out) *first_id_out = (uint32_t)s->materials.size();
  try {
    s->materials.insert(s->materials.end(), m, m + n);
  } catch (const std::bad_alloc&) {
    return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory");
  }
  return ZT_OK;
}

zt_status zt_scene_add_shapes(zt_scene* s, const zt_shape* shapes, size_t n) { /* Scene.add */
  if (!s || (!shapes && n)) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_add_shapes: NULL argument");
  for (size_t i = 0; i < n; ++i)
    if (shapes[i].kind > ZT_PLANE) return fail(ZT_ERR_INVALID_ARGUMENT, "unknown shape kind");
  release_staging(s);
  s->built = false; /* Scene.invalidate, scene.zig:98-102 */
  try {
    for (size_t i = 0; i < n; ++i) {
      if (shapes[i].kind == ZT_PLANE) s->planes.push_back(shapes[i]);
      else s->shapes.push_back(shapes[i]);
    }
  } catch (const std::bad_alloc&) {
    return fail(ZT_ERR_OUT_OF_MEMORY, "OutOfMemory");
  }
  return ZT_OK;
}

zt_status zt_scene_add_quad(zt_scene* s, const zt_vec3* c, const zt_vec3* u, const zt_vec3* v, uint32_t mat) {
  if (!s || !c || !u || !v) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_add_quad: NULL argument");
  /* scene.zig:82-88 */
  const double p1[3] = {c->x + u->x, c->y + u->y, c->z + u->z};
  const double p2[3] = {(c->x + u->x) + v->x, (c->y + u->y) + v->y, (c->z + u->z) + v->z};
  const double p3[3] = {c->x + v->x, c->y + v->y, c->z + v->z};
  zt_shape t[2];
  t[0].kind = t[1].kind = ZT_TRIANGLE;
  t[0].material = t[1].material = mat;
  const double c3[3] = {c->x, c->y, c->z};
  for (int k = 0; k < 3; ++k) {
    t[0].p[k] = c3[k]; t[0].p[3 + k] = p1[k]; t[0].p[6 + k] = p2[k];
    t[1].p[k] = c3[k]; t[1].p[3 + k] = p2[k]; t[1].p[6 + k] = p3[k];
  }
  return zt_scene_add_shapes(s, t, 2);
}

zt_status zt_scene_set_camera(zt_scene* s, const zt_camera_config* cfg) {
  if (!s || !cfg) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_set_camera: NULL argument");
  if (memcmp(&s->camera, cfg, sizeof *cfg) != 0) s->pilot_valid = false;
  s->camera = *cfg;
  return ZT_OK;
}

zt_status zt_scene_set_background(zt_scene* s, const zt_background* bg) {
  if (!s || !bg) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_set_background: NULL argument");
  if (bg->kind > ZT_BG_SKY) return fail(ZT_ERR_INVALID_ARGUMENT, "unknown background kind");
  if (memcmp(&s->background, bg, sizeof *bg) != 0) s->pilot_valid = false;
  s->background = *bg;
  return ZT_OK;
}

zt_status zt_scene_set_bvh(zt_scene* s, const zt_bvh_node* nodes, size_t n_nodes, const uint32_t* indices,
                           size_t n_indices) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_set_bvh: NULL scene");
  return import_bvh(s, nodes, n_nodes, indices, n_indices);
}

zt_status zt_scene_build(zt_scene* s) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_build: NULL scene");
  return build_scene(s);
}

zt_status zt_scene_build_device(zt_scene* s, uint32_t* used_device, double* build_ms) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_build_device: NULL scene");
  bool dev = false;
  const zt_status rc = build_scene(s, true, &dev, build_ms);
  if (used_device) *used_device = dev ? 1 : 0;
  return rc;
}

zt_status zt_scene_counts(const zt_scene* s, uint64_t* nm, uint64_t* nb, uint64_t* np, uint64_t* nn, uint64_t* nl) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_counts: NULL scene");
  if (nm) *nm = s->materials.size();
  if (nb) *nb = s->shapes.size();
  if (np) *np = s->planes.size();
  if (nn) *nn = s->nodes.size();
  if (nl) *nl = s->lights.size();
  return ZT_OK;
}

zt_status zt_scene_bvh(const zt_scene* s, zt_bvh_node* nodes, uint32_t* indices) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_bvh: NULL scene");
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built");
  for (size_t i = 0; nodes && i < s->nodes.size(); ++i) {
    const HostNode& h = s->nodes[i];
    nodes[i].bmin = zt_vec3{h.bmin[0], h.bmin[1], h.bmin[2]};
    nodes[i].bmax = zt_vec3{h.bmax[0], h.bmax[1], h.bmax[2]};
    nodes[i].first = h.first;
    nodes[i].count = h.count;
  }
  if (indices && !s->indices.empty()) memcpy(indices, s->indices.data(), s->indices.size() * sizeof(uint32_t));
  return ZT_OK;
}

zt_status zt_scene_lights(const zt_scene* s, zt_light* lights, double* cdf, double* total) {
  if (!s) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_lights: NULL scene");
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built");
  for (size_t i = 0; lights && i < s->lights.size(); ++i) {
    lights[i].shape = s->lights[i].shape;
    lights[i].radiance = zt_vec3{s->lights[i].radiance[0], s->lights[i].radiance[1], s->lights[i].radiance[2]};
    lights[i].weight = s->lights[i].weight;
  }
  if (cdf && !s->cdf.empty()) memcpy(cdf, s->cdf.data(), s->cdf.size() * sizeof(double));
  if (total) *total = s->total;
  return ZT_OK;
}

zt_status zt_scene_bvh_depth(const zt_scene* s, uint64_t* depth) {
  if (!s || !depth) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_scene_bvh_depth: NULL argument");
  if (!s->built) return fail(ZT_ERR_NOT_BUILT, "scene is not built");
  *depth = s->nodes.empty() ? 0 : depth_from(s, 0);
  return ZT_OK;
}

/* Output.encode / Image.toRgb8, image.zig:14-37, 65-73. */
zt_status zt_image_to_rgb8(const double* px, uint64_t n, uint32_t tonemap, double gamma, double exposure,
                           uint8_t* out) {
  if ((!px || !out) && n) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_image_to_rgb8: NULL argument");
  if (tonemap > 2) return fail(ZT_ERR_INVALID_ARGUMENT, "tonemap must be 0 (none), 1 (reinhard) or 2 (aces)");
  for (uint64_t i = 0; i < 3 * n; ++i) {
    const double v = isnan(px[i]) ? 0.0 : px[i];
    const double x = fmax(v * exposure, 0.0);
    double m;
    if (tonemap == 0) m = x;
    else if (tonemap == 1) m = x / (1.0 + x);
    else m = (x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14);
    const double mapped = fmax(0.0, fmin(m, 1.0));
    const double corrected = pow(mapped, 1.0 / gamma);
    out[i] = (uint8_t)round(fmax(0.0, fmin(corrected, 1.0)) * 255.0);
  }
  return ZT_OK;
}

const char* zt_last_error(void) { return g_last_error.c_str(); }
const char* zt_version(void) { return "zigtrace-b200 0.1.0"; }

}  /* extern "C" */

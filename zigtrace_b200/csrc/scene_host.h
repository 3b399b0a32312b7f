/*
 * scene_host.h -- host-side scene (src/scene.zig) with its binned-SAH BVH
 * (src/bvh.zig) and emitter table (src/light.zig), plus the flattening into
 * the device layout of zt_types.h.
 */
#ifndef ZT_SCENE_HOST_H
#define ZT_SCENE_HOST_H

#include <string>
#include <vector>

#include "../../include/zigtrace_b200.h"
#include "zt_types.h"

struct zt_device_buffers;  /* defined by the CUDA side */
struct zt_host_staging;    /* pinned flattened copy, defined by the CUDA side */

namespace zt {

struct HostNode {  /* Bvh.Node, bvh.zig:22-33 */
  double bmin[3], bmax[3];
  uint32_t first, count;
};

struct HostLight {  /* Light, light.zig:30-35 */
  zt_shape shape;
  double radiance[3];
  double weight;
};

/* Flattened arrays in the device layout (zt_types.h). */
struct FlatScene {
  std::vector<DPrim> prims;
  std::vector<int32_t> prim_ids;
  std::vector<DPair> pairs;
  std::vector<FPair> fpairs; /* conservative float copy of pairs (empty when the fast traversal cannot be used) */
  std::vector<DPrim> planes;
  std::vector<DMat> mats;
  std::vector<DLight> lights;
  std::vector<double> cdf;
  DevScene view;  /* pointers unset; counts, root, total, background set */
};

}  // namespace zt

struct zt_scene {
  std::vector<zt_material> materials;
  std::vector<zt_shape> shapes;  /* bounded, insertion order */
  std::vector<zt_shape> planes;  /* unbounded, insertion order */
  zt_camera_config camera;
  zt_background background;
  bool built = false;
  std::vector<zt::HostNode> nodes;
  std::vector<uint32_t> indices;
  std::vector<zt::HostLight> lights;
  std::vector<double> cdf;
  double total = 0;
  zt_device_buffers* device = nullptr;  /* resident copy, owned */
  bool pilot_valid = false;             /* mean_path is current for this build, camera and background */
  double mean_path = 0;                 /* mean path length of the pilot that ZT_MODE_AUTO reads */
  zt_host_staging* staging = nullptr;   /* pinned flattened copy, owned */
  uint64_t primal_cache_limit = 1ull << 30; /* bytes zt_forward may keep for zt_backward */
};

namespace zt {

void set_error(const std::string& msg);
zt_status fail(zt_status code, const std::string& msg);

/* Scene.build (scene.zig:92-96); with device = true the BVH is built on the
 * current CUDA device when it can be (see device_build_bvh), else on the
 * host.  *used_device tells which. */
zt_status build_scene(zt_scene* s, bool device = false, bool* used_device = nullptr, double* build_ms = nullptr);
/* Bvh.build on the current CUDA device (bvh_build.cu): the same nodes and
 * indices as the host build.  Returns ZT_DEVICE_BUILD_FALLBACK for input
 * the device build leaves to the host (splitMedian nodes, non-finite
 * boxes). */
constexpr zt_status ZT_DEVICE_BUILD_FALLBACK = 1;
zt_status device_build_bvh(zt_scene* s, double* build_ms);
/* Camera.init (camera.zig:29-55) for the given aspect ratio. */
DCamera camera_init(const zt_camera_config& cfg, double aspect);
/* Flattens a built scene into the device layout. */
void flatten_scene(const zt_scene* s, FlatScene* out);
/* Drops the resident device copy (implemented with the CUDA code). */
void release_device(zt_scene* s);
/* Drops the device copy and the pinned staging copy (scene changed). */
void release_staging(zt_scene* s);

}  // namespace zt

#endif

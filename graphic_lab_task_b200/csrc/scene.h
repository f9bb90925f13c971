// scene.h — host-side state of an lrt_scene (internal to liblrt_b200.so).
//
// The host arrays are exactly BVHRT's members (MultiRenderer/BVH2Common.h:
// 262-365); lrt_add_* fills them the way BVHRT's host code does
// (MultiRenderer/BVH2Common_host.cpp) and lrt_scene_upload replaces them
// wholesale.  The device copy and the derived device layouts live behind
// `dev` (device.cu).
#pragma once
#include <cstdint>
#include <string>
#include <map>
#include <vector>

#include "../../include/lrt_b200.h"
#include "device_layout.h"

namespace lrt {

struct DeviceScene; // device.cu

struct HostArrays {
  std::vector<lrt_bvh_node> nodesTLAS;
  std::vector<lrt_bvh_node_pair> allNodePairs;
  std::vector<lrt_instance_data> instanceData;
  std::vector<lrt_geom_data> geomData;
  std::vector<uint32_t> geomTags;
  std::vector<uint32_t> startEnd; // uint2 pairs, flattened
  std::vector<uint32_t> primIdCount;
  std::vector<uint32_t> indices;
  std::vector<float> vertPos; // float4 per vertex, flattened
  std::vector<uint32_t> primIndices;
  std::vector<lrt_bvh_node> origNodes;
  std::vector<lrt_sdf_frame_octree_node> sdfFrameOctreeNodes;
  std::vector<uint32_t> sdfFrameOctreeRoots;
  std::vector<lrt_sdf_svs_node> sdfSVSNodes;
  std::vector<uint32_t> sdfSVSRoots;
  std::vector<lrt_sdf_sbs_node> sdfSBSNodes;
  std::vector<uint32_t> sdfSBSData;
  std::vector<float> sdfSBSDataF;
  std::vector<uint32_t> sdfSBSRoots;
  std::vector<lrt_sdf_sbs_header> sdfSBSHeaders;
};

// Result of the structural validation that every upload goes through.
struct SceneInfo {
  uint32_t maxBlasDepth = 0;   // node pairs on the longest root-to-leaf path
  uint32_t tlasNodes = 0;
  bool hasTriangles = false, hasSbs = false, hasFrameOctree = false, hasSvs = false;
  bool hasSbsNeighbours = false; // SDF_SBS_NODE_LAYOUT_ID32F_IRGB32F_IN present
};

constexpr uint32_t kStartMask = 0x0FFFFFFFu;
constexpr uint32_t kSizeMask = 0x70000000u;
constexpr uint32_t kLeafNormal = 0xFFFFFFFFu;
constexpr uint32_t kEscapeRoot = 0xFFFFFFFEu;
constexpr uint32_t kMaxStack = 80; // STACK_SIZE, utils/raytracing/raytrace_common.h:36

inline uint32_t pack_offset_and_size(uint32_t start, uint32_t size)
{
  return kLeafBit | ((size << 28) & kSizeMask) | (start & kStartMask); // raytrace_common.h:51-54
}

} // namespace lrt

struct lrt_scene {
  lrt::HostArrays h;
  lrt_preset preset;
  uint32_t primsInLeaf = 2;
  uint32_t voxelStepCap = 0; // 0 = kMaxVoxelSteps
  bool committed = false;
  // geometry changes since the last full upload: a commit that finds none
  // re-uploads only the instances and the TLAS
  uint64_t geomVersion = 1;
  uint64_t uploadedGeomVersion = 0;
  uint64_t validatedGeomVersion = 0; // geometry arrays last passed validation at this version
  lrt::SceneInfo geomInfo;           // what that validation found
  lrt::SceneInfo info;
  lrt::DeviceScene* dev = nullptr;
  int device = -1;
  std::string err;
  uint64_t counters[LRT_COUNTER_COUNT] = {};
  // renderer materials (lrt_set_materials), validated; matVersion counts changes
  std::vector<lrt_material> mats;
  std::vector<uint32_t> matIds, matOffsets;
  uint64_t matVersion = 0;
  // renderer textures (lrt_set_textures: float4 texels of all images, width
  // and height of each, its first texel) and the triangle geometries' texture
  // coordinates (lrt_set_texcoords: 2 floats per vertex); texVersion counts changes
  std::vector<float> texels;
  std::vector<uint32_t> texDims;
  std::vector<uint64_t> texOffsets;
  std::map<uint32_t, std::vector<float>> texcoords;
  uint64_t texVersion = 0;
};

namespace lrt {
// scene.cpp
lrt_status validate(lrt_scene* s, SceneInfo* info);
lrt_status check_preset(lrt_scene* s, bool sphere_tracing_only = false);
lrt_status fail(lrt_scene* s, lrt_status code, const char* fmt, ...);
// device.cu
lrt_status device_upload(lrt_scene* s);
lrt_status device_update_instances(lrt_scene* s);
void device_release(lrt_scene* s);
} // namespace lrt

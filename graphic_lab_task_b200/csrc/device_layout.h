// device_layout.h — what the trace kernels read from HBM.
//
// The reference arrays are uploaded as-is where the kernels read them
// directly (TLAS nodes, BLAS node pairs, instances, leaf table, primIndices,
// SDF nodes, SBS data for hit colours).  Three derived layouts are built at
// upload for the B200 memory system:
//   * triSoup   — per reordered triangle {A, B-A, C-A} as 3 float4 (48 B, one
//                 128-B line per 2.7 triangles) instead of 3 index loads and 3
//                 dependent vertex gathers (BVH2Common.cpp:1580-1589);
//   * sbsDense  — every SBS brick resolved to a dense (brick_size+1)^3 fp32
//                 corner grid (2.9 KB for 8^3 bricks), so a voxel visit is 8
//                 loads from 4 adjacent 8-byte pairs instead of 8 index loads
//                 followed by 8 dependent value loads (BVH2Common.cpp:846-882);
//   * geoms     — 32 B per geometry with the tag, BLAS offset, leaf-table base
//                 and SDF ids the traversal needs (one load per BLAS entry).
// Values are copied bit for bit, so results do not depend on the layout.
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <vector_types.h>

#include "../../include/lrt_b200.h"

namespace lrt {

constexpr int kTraceThreads = 128;
// pixels of the tile one warp traces in lrt_trace_nearest_image (32 in all)
constexpr uint32_t kImgTileW = 8, kImgTileH = 4;

// Tile schedule of the image-order launches (one per stream and image size,
// two buffers used alternately): a header {longest tile cost, count of each
// of the kSchedClasses cost classes, warps of the launch, unused, 64-bit sum
// of the warps' busy times}, a bitmap of the listed tiles, one 64-bit cost
// accumulator per listed tile (the parts of a split tile add up there), then
// one list of `tiles` entries per class.  Everything before the lists is
// cleared before the launch that writes the buffer.  Costs are clock64 / 16.
constexpr uint32_t kSchedHeader = 8;
constexpr uint32_t kSchedWarps = 4;  // header word: warps that reported their busy time
constexpr uint32_t kSchedBusy = 6;   // header words 6-7: the sum of those busy times
constexpr uint32_t kSchedClasses = 3;
// When the previous launch was tail-bound (its longest tile took longer than
// its warps were busy on average), each tile of cost class 0 goes out as
// kSplitParts work items, each traced by one warp on 32 / kSplitParts of the
// tile's lanes (rows of the 8x4 tile): those tiles are the ones whose rays
// diverge most, and a warp serialises its lanes' divergent paths.
constexpr uint32_t kSplitParts = 2;
inline __host__ __device__ uint64_t sched_acc_offset(uint64_t tiles) // in words, 8-byte aligned
{
  return (kSchedHeader + (tiles + 31) / 32 + 1) & ~1ull;
}
inline __host__ __device__ uint64_t sched_lists_offset(uint64_t tiles)
{
  return sched_acc_offset(tiles) + 2 * tiles;
}
inline __host__ __device__ uint64_t sched_words(uint64_t tiles)
{
  return sched_lists_offset(tiles) + kSchedClasses * tiles;
}
// Per-thread shared-memory words after the traversal stack: the inputs of the
// deferred SDF normal (sign, sample point, 8 corner values), then those of the
// deferred SBS hit colour (object-space hit point, brick node index).
constexpr uint32_t kNormalWords = 16;
constexpr uint32_t kColourWord = 12;
// Dynamic shared memory of a trace kernel with stack_cap stack entries per thread.
constexpr size_t trace_smem_bytes(uint32_t stack_cap)
{
  return size_t(stack_cap + kNormalWords) * kTraceThreads * sizeof(uint32_t);
}
constexpr uint32_t kMaxStackDev = 80; // STACK_SIZE of raytrace_common.h:36
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kMaxVoxelSteps = 4096u; // voxel-march cap per brick (the reference loop is unbounded)

// preset-derived flags
constexpr uint32_t kFlagNeedNormal = 1u;
constexpr uint32_t kFlagStIterations = 2u;
constexpr uint32_t kFlagSurfaceMode = 4u; // REPRESENTATION_MODE_SURFACE
constexpr uint32_t kFlagBBoxMode = 8u;    // SDF_OCTREE_NODE_INTERSECT_BBOX
// every TLAS/BLAS node box has either no NaN coordinate or six (pruned pairs):
// node tests may use ray_box_nodes for rays with finite origin, direction and inverse
constexpr uint32_t kFlagCleanBoxes = 16u;
// bits 8..10: the preset's sdf_node_intersect (0 ST, 1 ANALYTIC, 2 NEWTON, 3 BBOX, 4 IT)
constexpr uint32_t kFlagSolverShift = 8u;
constexpr uint32_t kSolverST = 0, kSolverAnalytic = 1, kSolverNewton = 2, kSolverBBox = 3, kSolverIT = 4;

// error bits of the per-launch error word
constexpr uint32_t kErrStackOverflow = 1u;
constexpr uint32_t kErrVoxelCap = 2u;
constexpr uint32_t kErrLayerCap = 4u; // a transparency loop reached LRT_MAX_TRANSPARENCY_LAYERS

// work counters (same order as LRT_COUNTER_COUNT in lrt_b200.h)
enum : int {
  kCntTlasNodes = 0,
  kCntInstances,
  kCntBlasPairs,
  kCntLeafCalls,
  kCntTriTests,
  kCntBricks,
  kCntVoxels,
  kCntStSteps,
  kCntOctreeLeaves,
  kCntSvsLeaves,
  kCntHits,
  kCntNormals,
  kCntVoxelLoads
};

struct DevGeom {
  uint32_t tag;       // TAG_* (m_geomTags)
  uint32_t type;      // TYPE_* (GeomData.type)
  uint32_t bvhOffset; // first node pair of the BLAS
  uint32_t aabbBase;  // startEnd.x: base of this geometry's leaf table
  uint32_t triBase;   // triangles: GeomData.offset.x / 3
  uint32_t sdfId;     // SDF: GeomData.offset.x (index into roots/headers)
  uint32_t sdfRoot;   // SDF: root node index of this model
  uint32_t _pad;
};
static_assert(sizeof(DevGeom) == 32, "DevGeom is 32 bytes");

struct DevSbs {
  uint64_t denseBase;   // first float of node `root` in sbsDense
  uint32_t denseStride; // (brick_size+1)^3
  uint32_t brick_size;
  uint32_t v3;          // (brick_size + 2*pad + 1)^3
  uint32_t colorLayout; // 1 for the indexed ID32F layouts (hit colour from sbsDataF)
  uint32_t nodeCount;   // nodes of this model (leaves naming a node past it are skipped)
  uint32_t maskStride;  // words per brick in sbsMask: 1 + ceil(brick_size^3 / 32)
  uint64_t maskBase;    // first word of node `root` in sbsMask
  uint32_t pad;         // brick_pad
  uint32_t vsize;       // brick_size + 2*pad + 1
};

// sbsMask, per brick: word 0 is nonzero iff some voxel can start a sphere
// trace; words 1.. hold one bit per voxel (index (x*bs + y)*bs + z) that is
// set iff min of its 8 corner values <= 0 — the test OctreeBrickIntersect
// applies before LocalSurfaceIntersection (BVH2Common.cpp:941), evaluated on
// the same floats.  A clear bit means the reference does nothing in that
// voxel but advance the march.

typedef lrt_instance_data DevInstance;

// L2 prefetch of small scenes.  A launch whose rays are few takes as long as
// its slowest warp, a chain of dependent node, leaf and triangle loads; after
// an L2 flush (another job, a large previous launch) each of those is a DRAM
// round trip.  The trace kernel therefore streams the scene's node and leaf
// arrays into L2 first (cp.async.bulk.prefetch.L2, spread over its CTAs, one
// warp each), so that those chains run at L2 latency.  Ranges are taken in
// order while their sum stays within kPrefetchMaxBytes (well inside the
// 126 MB L2, leaving room for rays and hits); launches of fewer than
// kPrefetchMinRays rays skip it.
constexpr int kPrefetchRanges = 10;
constexpr uint64_t kPrefetchMaxBytes = 48ull << 20;
constexpr uint64_t kPrefetchMinRays = 4096;
constexpr uint32_t kPrefetchChunk = 4096; // bytes per prefetch instruction

struct DevScene {
  const lrt_bvh_node* tlas;
  const lrt_bvh_node_pair* pairs;
  const DevInstance* instances;
  const DevGeom* geoms;
  const uint32_t* primIdCount;
  const float4* triSoup;
  const uint32_t* primIndices;
  const lrt_bvh_node* origNodes;
  const lrt_sdf_frame_octree_node* frameOctreeNodes;
  const lrt_sdf_svs_node* svsNodes;
  const lrt_sdf_sbs_node* sbsNodes;
  const uint32_t* sbsData;
  const float* sbsDataF;
  const float* sbsDense;
  const uint32_t* sbsMask;
  const DevSbs* sbs;
  uint32_t flags;
  uint32_t voxelStepCap; // bounded SBS voxel march (kMaxVoxelSteps unless set)
  // byte ranges streamed into L2 at the start of a trace launch (16-byte
  // aligned bases, sizes multiples of 16; 0 bytes: none)
  const char* pfPtr[kPrefetchRanges];
  uint64_t pfBytes[kPrefetchRanges];
};

struct DevCamera {
  float proj_inv[16];
  float world_view_inv[16];
  uint32_t width, height;
  float tnear, tfar;
};

// Lights and background of the fused camera render (lrt_light is Light of
// core/IRenderer.h:72-78).
typedef lrt_light DevLight;
struct DevLights {
  DevLight light[LRT_MAX_LIGHTS];
  uint32_t count;
  float background[4];
};

// The renderer's material tables for the transparency loop (lrt_material =
// MultiRendererMaterial, core/IRenderer.h:31-38; offsets = uint2 {start,
// size} per geometry) and the background colour.
struct DevMaterials {
  const lrt_material* mats;
  const uint32_t* ids;
  const uint2* offsets;
  float background[4];
  // the renderer's textures (MultiRenderer::m_textures): texels, and per
  // texture {first texel, width, height, 0}; the texture coordinates of each
  // triangle slot's 3 vertices (the triangle soup's indexing), or NULL
  const float4* texels;
  const uint4* texs;
  uint32_t texCount;
  const float2* triTc;
};

// The render mode of lrt_render_rgba8's general kernel: the preset's
// render_mode, its sample count (initEyeRay's sqrt(spp) grid, or one point
// for RAY_GEN_MODE_RANDOM) and whether the transparency path applies.
struct DevRenderModes {
  uint32_t mode;
  uint32_t samples;
  uint32_t sqrtSpp;
  float invSqrt;
  uint32_t random;
  float randomX, randomY;
  uint32_t transparency;
};

// One camera of a batched multi-camera trace: its rays are generated in the
// kernel, tile by tile; hits go to out[rayOffset + y*width + x].
struct DevBatchCamera {
  DevCamera cam;
  uint64_t rayOffset;
  uint32_t tileBase; // first global tile index of this camera
  uint32_t tilesX;   // tiles per image row
};

// Launch shape of the batched trace, chosen by the autotuner: tiles of
// tileW x tileH pixels (tileW*tileH = 32*raysPerLane) fetched by one warp at
// a time; each lane traces raysPerLane pixels of its tile one after another.
struct DevBatchShape {
  uint32_t tileW, tileH, raysPerLane, stackCap;
};

} // namespace lrt

/*
 * lrt_b200.h — C-ABI of the B200 ray-query library (liblrt_b200.so).
 *
 * The library replaces LiteRT's CPU/Vulkan implementation of
 * BVHRT::RayQuery_NearestHit (MultiRenderer/BVH2Common.cpp:3322-3392) with
 * hand-written sm_100a CUDA kernels.  Every entry point takes plain pointers
 * and sizes; no C++ or torch type crosses this boundary.
 *
 * Data layouts below are byte-for-byte the reference's device-visible structs
 * (the arrays that kernel1D_FillGbuffer.slang:6-50 binds), so a BVHRT that was
 * filled by the reference's own host code can be uploaded unchanged.
 *
 * Conventions
 *  - Every function returns an lrt_status; nothing aborts.  On failure the
 *    scene keeps a message readable with lrt_last_error().
 *  - A scene is confined to one host thread at a time.  Concurrent traces of
 *    one scene go through different CUDA streams.
 *  - Host pointers passed to lrt_add_* / lrt_scene_upload are copied before
 *    the call returns (reference ownership rule, BVH2Common_host.cpp:317-327).
 */
#ifndef LRT_B200_H
#define LRT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                             */
/* ------------------------------------------------------------------------ */
typedef int32_t lrt_status;
enum {
  LRT_OK = 0,
  LRT_ERR_INVALID_ARGUMENT = 1,  /* null pointer, bad id, bad size          */
  LRT_ERR_BAD_SCENE = 2,         /* uploaded arrays fail validation          */
  LRT_ERR_NOT_COMMITTED = 3,     /* trace before CommitScene / upload        */
  LRT_ERR_CUDA = 4,              /* a CUDA runtime call failed               */
  LRT_ERR_DEVICE_LIMIT = 5,      /* kernel reported a bounded-loop limit     */
  LRT_ERR_UNSUPPORTED = 6,       /* preset or layout outside the hot path    */
  LRT_ERR_OUT_OF_MEMORY = 7
};

/* ------------------------------------------------------------------------ */
/* Reference PODs (same sizes, field order and meaning)                     */
/* ------------------------------------------------------------------------ */

/* CRT_Hit, CrossRT/CrossRT.h:26-33 (32 bytes). */
typedef struct lrt_hit {
  float t;
  uint32_t primId;
  uint32_t instId;
  uint32_t geomId; /* type << 24 | geometry id */
  float coords[4];
} lrt_hit;

/* BVHNode, utils/raytracing/cbvh.h:21-27 (32 bytes). */
typedef struct lrt_bvh_node {
  float boxMin[3];
  uint32_t leftOffset; /* LEAF_BIT 0x80000000 marks a leaf */
  float boxMax[3];
  uint32_t escapeIndex;
} lrt_bvh_node;

/* BVHNodePair, utils/raytracing/cbvh.h:29-33 (64 bytes). */
typedef struct lrt_bvh_node_pair {
  lrt_bvh_node left;
  lrt_bvh_node right;
} lrt_bvh_node_pair;

/* GeomData, utils/raytracing/intersection_common.h:33-44 (64 bytes). */
typedef struct lrt_geom_data {
  float boxMin[4];
  float boxMax[4];
  uint32_t bvhOffset;
  uint32_t type;      /* TYPE_* of core/render_settings.h */
  uint32_t offset[2]; /* triangles: (index offset, vertex offset); SDF: (sdf id, 0) */
  uint32_t hasChannels;
  uint32_t _pad[3];
} lrt_geom_data;

/* InstanceData, utils/raytracing/intersection_common.h:47-56 (256 bytes).
 * Matrices are LiteMath float4x4: column-major, element (row r, col c) at
 * [c*4 + r]. */
typedef struct lrt_instance_data {
  float boxMin[4];
  float boxMax[4];
  uint32_t geomId;
  uint32_t _pad[7];
  float transform[16];
  float transformInv[16];
  float transformInvTransposed[16];
} lrt_instance_data;

/* SdfFrameOctreeNode, sdf/simple/sdf_simple_shared.h:23-27 (36 bytes). */
typedef struct lrt_sdf_frame_octree_node {
  float values[8];
  uint32_t offset; /* children start (8 consecutive nodes); 0 = leaf */
} lrt_sdf_frame_octree_node;

/* SdfSVSNode, sdf/simple/sdf_simple_shared.h:30-35 (16 bytes). */
typedef struct lrt_sdf_svs_node {
  uint32_t pos_xy;
  uint32_t pos_z_lod_size;
  uint32_t values[2]; /* 8 x u8 quantised distances */
} lrt_sdf_svs_node;

/* SdfSBSNode, sdf/simple/sdf_simple_shared.h:39-45 (16 bytes). */
typedef struct lrt_sdf_sbs_node {
  uint32_t pos_xy;
  uint32_t pos_z_lod_size;
  uint32_t data_offset; /* in uint32 words of the SBS data array */
  uint32_t _pad;
} lrt_sdf_sbs_node;

/* SdfSBSHeader, sdf/simple/sdf_simple_shared.h:49-55 (16 bytes). */
typedef struct lrt_sdf_sbs_header {
  uint32_t brick_size;
  uint32_t brick_pad;
  uint32_t bytes_per_value;
  uint32_t aux_data; /* SDF_SBS_NODE_LAYOUT_* */
} lrt_sdf_sbs_header;

/* MultiRenderPreset, core/render_settings.h:116-137 (60 bytes). */
typedef struct lrt_preset {
  uint32_t render_mode;
  uint32_t sdf_node_intersect; /* SDF_OCTREE_NODE_INTERSECT_*: 0 ST, 1 ANALYTIC, 2 NEWTON, 3 BBOX, 4 IT (render_settings.h:54-58) */
  uint32_t normal_mode;
  uint32_t ray_gen_mode;
  uint32_t interpolation_mode;
  uint32_t representation_mode;
  uint32_t spp;
  uint32_t fixed_lod;
  float level_of_detail;
  float compact_sdf_eps;
  float LOD_distance;
  uint32_t channel_render_mode;
  uint32_t channel_id;
  uint32_t component_id;
  uint32_t CTF_id;
} lrt_preset;

/* Constants of the reference the C-ABI exposes. */
#define LRT_TYPE_MESH_TRIANGLE 0u  /* core/render_settings.h:4 */
#define LRT_TYPE_SDF_FRAME_OCTREE 3u
#define LRT_TYPE_SDF_SVS 5u
#define LRT_TYPE_SDF_SBS 6u
#define LRT_TYPE_SDF_SBS_TEX 10u
#define LRT_TYPE_SDF_SBS_COL 11u
#define LRT_TYPE_GRAPHICS_PRIM 17u
#define LRT_TAG_NONE 0u            /* MultiRenderer/BVH2Common.h:30-43 */
#define LRT_TAG_TRIANGLE 1u
#define LRT_TAG_SDF_BRICK 4u
#define LRT_TAG_SDF_NODE 8u
#define LRT_SBS_LAYOUT_UNDEFINED (0u << 24)  /* sdf_simple_shared.h:12-20 */
#define LRT_SBS_LAYOUT_DX (1u << 24)
#define LRT_SBS_LAYOUT_DX_UV16 (2u << 24)
#define LRT_SBS_LAYOUT_DX_RGB8 (3u << 24)
#define LRT_SBS_LAYOUT_ID32F_IRGB32F (4u << 24)
#define LRT_SBS_LAYOUT_ID32F_IRGB32F_IN (5u << 24)
#define LRT_SBS_LAYOUT_MASK 0xFF000000u
#define LRT_RENDER_MODE_LAMBERT_NO_TEX 1u
#define LRT_RENDER_MODE_ST_ITERATIONS 10u
#define LRT_RENDER_MODE_OUTLINE_PRIM 13u   /* MULTI_RENDER_MODE_*, core/render_settings.h */
#define LRT_RENDER_MODE_OUTLINE_BORDER 14u
#define LRT_SDF_INTERSECT_ST 0u
#define LRT_NORMAL_MODE_GEOMETRY 0u
#define LRT_INTERPOLATION_TRILINEAR 0u
#define LRT_REPRESENTATION_VOLUME 1u

/* ------------------------------------------------------------------------ */
/* Scene object (ISceneObject, CrossRT/CrossRT.h:43-175)                    */
/* ------------------------------------------------------------------------ */
typedef struct lrt_scene lrt_scene;

/* CreateSceneRT("BVH2Common_B200", build, layout)
 * (BVH2Common_host.cpp:1594-1600).  build_name follows the reference's
 * BuilderPresetsFromString: a trailing digit sets primitives per triangle
 * leaf ("cbvh_embree2" -> 2).  Either name may be NULL. */
lrt_status lrt_scene_create(const char* build_name, const char* layout_name, lrt_scene** out);
lrt_status lrt_scene_destroy(lrt_scene* scene);

/* Message of the last failed call on this scene (or of the last failed
 * lrt_scene_create when scene is NULL).  Never NULL. */
const char* lrt_last_error(const lrt_scene* scene);

/* BVHRT::SetPreset (BVH2Common_host.cpp:1437-1454).  Takes effect for the
 * next trace; no recommit needed. */
lrt_status lrt_set_preset(lrt_scene* scene, const lrt_preset* preset);
/* getDefaultPreset() (core/render_settings.h:139-160). */
lrt_status lrt_default_preset(lrt_preset* out);

/* ISceneObject::ClearGeom (CrossRT.h:60; BVH2Common_host.cpp:128-156). */
lrt_status lrt_clear_geom(lrt_scene* scene);

/* Build qualities of the reference's BuildOptions (CrossRT/CrossRT.h:14-17).
 * LRT_BUILD_LOW builds the tree on the current CUDA device (a linear BVH over
 * Morton-sorted box centres, Karras 2012) instead of the host's binned SAH:
 * orders of magnitude faster for large meshes, with the same array formats
 * and a tree that traverses somewhat slower.  It needs a CUDA device (else
 * LRT_ERR_CUDA) and takes effect in lrt_add_geom_triangles3f,
 * lrt_add_geom_aabb and, for the TLAS, lrt_commit_scene.  The other values
 * select the SAH build. */
#define LRT_BUILD_LOW 0x1u
#define LRT_BUILD_MEDIUM 0x2u
#define LRT_BUILD_HIGH 0x4u
#define LRT_BUILD_REFIT 0x8u

/* ISceneObject::AddGeom_Triangles3f (CrossRT.h:71-72;
 * BVH2Common_host.cpp:307-359).  vertex_byte_stride 0 means 12. */
lrt_status lrt_add_geom_triangles3f(lrt_scene* scene, const float* vpos3f, size_t vert_count,
                                    const uint32_t* tri_indices, size_t index_count, uint32_t build_flags,
                                    size_t vertex_byte_stride, uint32_t* geom_id_out);

/* ISceneObject::AddGeom_AABB (CrossRT.h:95; BVH2Common_host.cpp:441-459).
 * boxes: n x {float4 boxMin, float4 boxMax}.  Like the reference, this adds
 * the BLAS and its leaf table only; the SDF adders below call it. */
lrt_status lrt_add_geom_aabb(lrt_scene* scene, uint32_t type_tag, const float* boxes_min_max_f8,
                             size_t box_count, uint32_t build_flags, uint32_t* geom_id_out);

/* BVHRT::AddGeom_SdfFrameOctree (BVH2Common_host.cpp:501-534). */
lrt_status lrt_add_geom_sdf_frame_octree(lrt_scene* scene, const lrt_sdf_frame_octree_node* nodes,
                                         size_t node_count, uint32_t* geom_id_out);
/* BVHRT::AddGeom_SdfSVS (BVH2Common_host.cpp:536-599). */
lrt_status lrt_add_geom_sdf_svs(lrt_scene* scene, const lrt_sdf_svs_node* nodes, size_t node_count,
                                uint32_t* geom_id_out);
/* BVHRT::AddGeom_SdfSBS (BVH2Common_host.cpp:601-695).  values_f may be NULL
 * for the DX layouts. */
lrt_status lrt_add_geom_sdf_sbs(lrt_scene* scene, const lrt_sdf_sbs_header* header,
                                const lrt_sdf_sbs_node* nodes, size_t node_count, const uint32_t* values,
                                size_t values_count, const float* values_f, size_t values_f_count,
                                uint32_t* geom_id_out);

/* ISceneObject::ClearScene / AddInstance / CommitScene (CrossRT.h:101-115;
 * BVH2Common_host.cpp:1230-1301).  matrix: 16 floats, column-major.
 * CommitScene builds the TLAS and uploads everything to the current device. */
/* The same adders reading the reference's model files (sdf/simple/
 * sdf_simple.cpp:50-142): frame octree and SVS = u32 node count + nodes; SBS
 * = header, u32 node count, nodes, u32 value count, values, u32 float count,
 * floats (older files end after the values).  Files shorter than their counts
 * are refused with LRT_ERR_INVALID_ARGUMENT. */
lrt_status lrt_add_geom_sdf_frame_octree_file(lrt_scene* scene, const char* path, uint32_t* geom_id_out);
lrt_status lrt_add_geom_sdf_svs_file(lrt_scene* scene, const char* path, uint32_t* geom_id_out);
lrt_status lrt_add_geom_sdf_sbs_file(lrt_scene* scene, const char* path, uint32_t* geom_id_out);

lrt_status lrt_clear_scene(lrt_scene* scene);
lrt_status lrt_add_instance(lrt_scene* scene, uint32_t geom_id, const float* matrix_col_major16,
                            uint32_t* inst_id_out);
/* build_flags may include LRT_COMMIT_HOST_ONLY: build the TLAS and validate,
 * but leave the device untouched (for a host that hands the arrays to another
 * implementation through lrt_scene_export). */
#define LRT_COMMIT_HOST_ONLY 0x100u
lrt_status lrt_commit_scene(lrt_scene* scene, uint32_t build_flags);

/* ISceneObject::UpdateInstance (CrossRT.h:116; BVHRT::UpdateInstance,
 * MultiRenderer/BVH2Common_host.cpp:1303-1335): the new column-major
 * transform of instance inst_id, its box recomputed from the geometry's box;
 * it takes effect at the next lrt_commit_scene, which rebuilds the TLAS and,
 * when no geometry changed since the last upload, writes only the TLAS and
 * the instances to the device.  As in the reference, transformInvTransposed
 * (the normal matrix) keeps its old value unless LRT_UPDATE_NORMAL_MATRIX is
 * set; inst_id must be below the instance count (the reference also accepts
 * the count itself and writes past its array). */
#define LRT_UPDATE_NORMAL_MATRIX 0x1u
lrt_status lrt_update_instance(lrt_scene* scene, uint32_t inst_id, const float* matrix_col_major16, uint32_t flags);

/* ------------------------------------------------------------------------ */
/* Drop-in upload of arrays flattened by the reference's BVHRT host code.     */
/* ------------------------------------------------------------------------ */
/* One {pointer, element count} per BVHRT member the traversal reads
 * (MultiRenderer/BVH2Common.h:262-365).  startEnd holds uint2 pairs and
 * vertPos float4s: their counts are in pairs / float4s. */
typedef struct lrt_scene_arrays {
  const lrt_bvh_node* nodesTLAS;                        uint64_t nodesTLAS_count;
  const lrt_bvh_node_pair* allNodePairs;                uint64_t allNodePairs_count;
  const lrt_instance_data* instanceData;                uint64_t instanceData_count;
  const lrt_geom_data* geomData;                        uint64_t geomData_count;
  const uint32_t* geomTags;                             uint64_t geomTags_count;
  const uint32_t* startEnd;                             uint64_t startEnd_count;
  const uint32_t* primIdCount;                          uint64_t primIdCount_count;
  const uint32_t* indices;                              uint64_t indices_count;
  const float* vertPos;                                 uint64_t vertPos_count;
  const uint32_t* primIndices;                          uint64_t primIndices_count;
  const lrt_bvh_node* origNodes;                        uint64_t origNodes_count;
  const lrt_sdf_frame_octree_node* sdfFrameOctreeNodes; uint64_t sdfFrameOctreeNodes_count;
  const uint32_t* sdfFrameOctreeRoots;                  uint64_t sdfFrameOctreeRoots_count;
  const lrt_sdf_svs_node* sdfSVSNodes;                  uint64_t sdfSVSNodes_count;
  const uint32_t* sdfSVSRoots;                          uint64_t sdfSVSRoots_count;
  const lrt_sdf_sbs_node* sdfSBSNodes;                  uint64_t sdfSBSNodes_count;
  const uint32_t* sdfSBSData;                           uint64_t sdfSBSData_count;
  const float* sdfSBSDataF;                             uint64_t sdfSBSDataF_count;
  const uint32_t* sdfSBSRoots;                          uint64_t sdfSBSRoots_count;
  const lrt_sdf_sbs_header* sdfSBSHeaders;              uint64_t sdfSBSHeaders_count;
} lrt_scene_arrays;

/* Replace the scene's host arrays with copies of `arrays`, validate them and
 * upload to the current device.  Equivalent of the reference GPU class's
 * CommitDeviceData (MultiRenderer_slang_comp.cpp:264). */
lrt_status lrt_scene_upload(lrt_scene* scene, const lrt_scene_arrays* arrays);

/* Read-only view of the scene's host arrays (valid until the next mutating
 * call).  Lets a host that built the scene with lrt_add_* hand the same
 * arrays to another implementation. */
lrt_status lrt_scene_export(const lrt_scene* scene, lrt_scene_arrays* out);

/* ------------------------------------------------------------------------ */
/* Ray queries                                                              */
/* ------------------------------------------------------------------------ */
/* Flags for the trace calls. */
#define LRT_TRACE_DEVICE_POINTERS 0x1u /* rays/hits are device pointers     */
#define LRT_TRACE_FAST_MATH 0x2u       /* FMA-contracted kernels (tolerance
                                          parity); default is the exact build */
#define LRT_TRACE_COUNT_WORK 0x4u      /* also accumulate work counters     */
#define LRT_TRACE_NATURAL_ORDER 0x8u   /* image-order calls and large device-
                                          pointer traces: no tile schedule */

/* Batched BVHRT::RayQuery_NearestHit.  rays: n x {float4 posAndNear,
 * float4 dirAndFar} (32 bytes per ray), hits: n x lrt_hit.  A ray whose
 * dirAndFar.w <= 0 is traced stop-on-first-hit with tfar = -w, exactly like
 * the reference (BVH2Common.cpp:3324-3326).  stream is a cudaStream_t (NULL =
 * legacy default stream).  With host pointers the call is synchronous.  A
 * warp traces 32 consecutive rays; a device-pointer trace of fewer rays than
 * the GPU holds warps gives each warp 16 or 8 rays strided across the call,
 * and one of more rays that repeats the previous device-pointer trace's ray
 * count on the stream hands its 32-ray groups out in a schedule kept per
 * stream and ray count, as lrt_trace_nearest_image does with its tiles
 * (slowest groups first; LRT_TRACE_NATURAL_ORDER turns it off).  The order
 * never changes a hit. */
lrt_status lrt_trace_nearest(lrt_scene* scene, const float* rays, lrt_hit* hits, uint64_t n, void* stream,
                             uint32_t flags);

/* Allocation-free variant of lrt_trace_nearest.  No counterpart in the
 * reference: it exists for hosts that cannot call cudaMalloc once their scene
 * is uploaded (an application that gives its whole GPU memory budget to its
 * own pool, or forbids device allocation inside its frame loop).  The trace
 * kernel's scratch (ray counter, error word) and, for host buffers, the
 * staging copies of rays and hits live in a fixed file-scope device array of
 * 1 MiB + 256 B, which a GPU holds from the first scene upload on it until
 * the process exits: the upload (lrt_commit_scene, lrt_scene_upload) looks
 * the array's device address up with the scene's device current, so this
 * call loads no module and allocates no device memory.  With host pointers at
 * most 16384 rays per call are accepted (larger n returns
 * LRT_ERR_INVALID_ARGUMENT); with LRT_TRACE_DEVICE_POINTERS any n.  The call
 * calls no cudaMalloc/cudaFree and is synchronous: it returns after `stream`
 * has drained, with LRT_ERR_DEVICE_LIMIT if the kernel hit a bounded-loop
 * limit.  The scene's device must be current.  All calls share the one
 * array: calls that overlap on the GPU (different streams, threads or scenes
 * on one device) race and must be serialised by the caller.
 * LRT_TRACE_COUNT_WORK is not supported. */
lrt_status lrt_trace_nearest_noalloc(lrt_scene* scene, const float* rays, lrt_hit* hits, uint64_t n, void* stream,
                                     uint32_t flags);

/* Waits for the traces queued on `stream` (device-pointer traces are
 * asynchronous) and returns LRT_ERR_DEVICE_LIMIT if one of them hit a
 * bounded-loop limit.  With read_counters != 0 the work counters of the last
 * LRT_TRACE_COUNT_WORK trace on the stream become readable. */
lrt_status lrt_trace_sync(lrt_scene* scene, void* stream, int32_t read_counters);

/* lrt_trace_nearest for the width*height rays of one image stored in
 * row-major pixel order, device pointers only (asynchronous on `stream`,
 * flags: LRT_TRACE_FAST_MATH, LRT_TRACE_COUNT_WORK, LRT_TRACE_NATURAL_ORDER).
 * A warp traces an 8x4 tile of pixels rather than 32 pixels of one row, as
 * the reference's kernel1D_FillGbuffer walks pixels in packed tiles
 * (MultiRenderer.cpp:185-202); every hit equals lrt_trace_nearest's for the
 * same ray.  Tiles are scheduled longest first: each launch measures its
 * tiles' durations, and the next launch of the same image size on the same
 * stream starts with the tiles that took at least 1/2, then 1/4, then 1/8 of
 * the longest (the rest follow in row order), so that a few slow tiles do
 * not finish last; when the longest tile took longer than the warps were
 * busy on average, the tiles of the first group are each traced by two warps
 * (two rows of the tile each).  The order never changes a result; the first
 * launch of a size on a stream allocates that stream's two schedule buffers
 * (about 36 bytes + 20.1 bytes per tile each).  lrt_render_rgba8,
 * lrt_fill_gbuffer_transparency and the _image forms of the Lambert passes
 * schedule their tiles the same way.  No counterpart entry point in the
 * reference. */
lrt_status lrt_trace_nearest_image(lrt_scene* scene, const float* rays_dev, lrt_hit* hits_dev, uint32_t width,
                                   uint32_t height, void* stream, uint32_t flags);

/* ISceneObject::RayQuery_NearestHit / RayQuery_AnyHit for one ray
 * (CrossRT.h:145,163).  Synchronous; forwards to a 1-ray batch. */
lrt_status lrt_ray_query_nearest_hit(lrt_scene* scene, const float pos_and_near[4], const float dir_and_far[4],
                                     lrt_hit* hit_out);
lrt_status lrt_ray_query_any_hit(lrt_scene* scene, const float pos_and_near[4], const float dir_and_far[4],
                                 int32_t* hit_out);

/* Iteration cap of the SBS voxel march per brick (default 4096).  The
 * reference loop (BVH2Common.cpp:919-1032) has no cap; a ray that reaches
 * the cap stops marching that brick and the trace returns
 * LRT_ERR_DEVICE_LIMIT instead of hanging.  0 restores the default. */
lrt_status lrt_set_voxel_step_limit(lrt_scene* scene, uint32_t steps);

/* Work counters of the last LRT_TRACE_COUNT_WORK trace (summed over rays):
 * TLAS node visits, instances entered, BLAS node-pair visits, leaf calls,
 * triangle tests, SBS brick entries, SBS voxel-march iterations, ST steps,
 * frame-octree leaf tests, SVS leaf tests, hits, normals computed, and SBS
 * voxels whose 8 corner values were loaded to start a sphere trace.  The
 * kernels never enter SBS subtrees or bricks that hold no voxel able to start
 * a sphere trace, so their node-pair, leaf-call, brick and voxel-march counts
 * are at most the reference algorithm's; every other counter equals it. */
#define LRT_COUNTER_COUNT 13
lrt_status lrt_get_work_counters(lrt_scene* scene, uint64_t counters[LRT_COUNTER_COUNT]);

/* ------------------------------------------------------------------------ */
/* Eye rays (MultiRenderer::initEyeRay, MultiRenderer.cpp:142-183)           */
/* ------------------------------------------------------------------------ */
/* One pinhole camera: the inverses of the projection and world-view matrices
 * (column-major), the image size and the ray interval.  Rays are generated
 * for pixel centres (spp = 1, frame 0); the cutting plane is off, so the
 * reference would use tnear = 1e-9 and tfar = 1e9. */
typedef struct lrt_camera {
  float proj_inv[16];
  float world_view_inv[16];
  uint32_t width;
  uint32_t height;
  float tnear;
  float tfar;
} lrt_camera;

/* Write width*height rays of `camera` (row-major pixel order) to device
 * memory `rays_dev`. */
lrt_status lrt_generate_eye_rays(lrt_scene* scene, const lrt_camera* camera, float* rays_dev, void* stream);

/* One cosine-weighted diffuse bounce ray per ray of a traced batch (a second
 * wavefront): origin at the hit point, direction from
 * MapSampleToCosineDistribution with power 1 (utils/raytracing/
 * render_common.h:75-113) around the hit's decoded normal turned towards the
 * incoming ray, two uniforms from a PCG hash of (ray index, seed), interval
 * [tnear, tfar].  Rays whose primary ray missed get a NaN origin (a NaN ray
 * misses everything; callers may drop them).  All buffers are device memory,
 * 16-byte aligned; asynchronous on `stream`. */
lrt_status lrt_generate_bounce_rays(lrt_scene* scene, const float* rays_dev, const lrt_hit* hits_dev, uint64_t n,
                                    uint64_t seed, float tnear, float tfar, float* bounce_rays_dev, void* stream);

/* lrt_generate_bounce_rays without the rays whose primary ray missed: the
 * bounce rays of the hits, in increasing order of the traced ray, packed
 * into bounce_dev[0 .. *count_dev), with index_dev[k] the traced ray of
 * bounce ray k (each bounce ray equals lrt_generate_bounce_rays's for that
 * ray).  count_dev: one uint64 in device memory, written on `stream` (read it
 * back, or size the next trace by it).  At most 2^32 - 1 rays.  Three
 * launches (count per tile, scan, write), no host synchronisation.  The
 * per-tile counts live in scratch kept with the scene: calls that overlap on
 * different streams race. */
lrt_status lrt_generate_bounce_rays_compact(lrt_scene* scene, const float* rays_dev, const lrt_hit* hits_dev,
                                            uint64_t n, uint64_t seed, float tnear, float tfar, float* bounce_dev,
                                            uint32_t* index_dev, uint64_t* count_dev, void* stream);

/* lrt_generate_bounce_rays_compact with the bounce rays in coherence order
 * instead of ray order, so that a warp's 32 rays head the same way from
 * nearby points: sorted (stably, ties in ray order) by the key
 *   min(cell(d.x) << 22 | cell(d.y) << 20 | cell(d.z) << 18
 *       | morton(q.x, q.y, q.z), 2^24 - 2)
 * of the bounce direction d and origin o, with cell(v) = clamp(int((v + 1) *
 * 2), 0, 3), q = clamp(int((o - lo) * (64 / (hi - lo))), 0, 63) per axis
 * over the union [lo, hi] of the instances' world boxes (float32, each
 * operation rounded to nearest), and morton() interleaving the three 6-bit
 * values x-highest.  index_dev[k] is the traced ray of bounce ray k;
 * index_dev must hold n entries (its entries from *count_dev on are
 * unspecified), as must bounce_dev.  At most 2^31 - 1 rays.  Three launches
 * plus a device radix sort, no host synchronisation; the scratch grows with
 * n on the device and is kept with the scene, so calls that overlap on
 * different streams race.  Each bounce ray equals
 * lrt_generate_bounce_rays's for its traced ray. */
lrt_status lrt_generate_bounce_rays_sorted(lrt_scene* scene, const float* rays_dev, const lrt_hit* hits_dev,
                                           uint64_t n, uint64_t seed, float tnear, float tfar, float* bounce_dev,
                                           uint32_t* index_dev, uint64_t* count_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* Differentiable form (SBS distances)                                      */
/* ------------------------------------------------------------------------ */
/* No counterpart exists in the reference (its differentiable renderer
 * sources are absent).  A Lambert image of n rays (device memory, 32 B per
 * ray) is rendered through the same traversal as lrt_trace_nearest:
 * image[i] = max(0, n_i . light) for the nearest hit's decoded normal
 * (MultiRenderer_resolve.cpp:617-666 for LAMBERT_NO_TEX, one directional
 * light of unit colour, albedo 1), 0 for misses.  Asynchronous on `stream`;
 * lrt_trace_sync(stream) reports bounded-loop limits.  A call of a wave or
 * more of rays that repeats the previous device trace's ray count on the
 * stream (an optimisation loop) hands its 32-ray groups out in the stream's
 * schedule for that count, as lrt_trace_nearest does; the pixels are the
 * same, the gradient's atomic additions come in another order. */
lrt_status lrt_render_lambert(lrt_scene* scene, const float* rays_dev, uint64_t n, const float light[3],
                              float* image_dev, void* stream);

/* lrt_render_lambert for rays that form a width x height image (row-major
 * pixels; several views of one size stack as a taller image), traced in
 * 8x4-pixel tiles per warp in the stream's longest-first tile schedule, which
 * it shares with lrt_trace_nearest_image, lrt_render_rgba8 and
 * lrt_adjoint_lambert_sbs_image (LRT_TRACE_NATURAL_ORDER, the only flag:
 * tiles in row order).  Every pixel's value equals lrt_render_lambert's. */
lrt_status lrt_render_lambert_image(lrt_scene* scene, const float* rays_dev, uint32_t width, uint32_t height,
                                    const float light[3], float* image_dev, void* stream, uint32_t flags);

/* Light, core/IRenderer.h:72-78 (32 bytes).  space is the direction of a
 * LRT_LIGHT_DIRECT light (normalised by the caller, as create_direct_light
 * does) or the position of a LRT_LIGHT_POINT one; color includes intensity. */
typedef struct lrt_light {
  float space[3];
  uint32_t type; /* LIGHT_TYPE_*, core/IRenderer.h:16-18 */
  float color[3];
  uint32_t _pad;
} lrt_light;
enum { LRT_LIGHT_DIRECT = 0, LRT_LIGHT_POINT = 1, LRT_LIGHT_AMBIENT = 2 };
#define LRT_MAX_LIGHTS 16

/* MultiRenderer::Render (MultiRenderer.cpp:14-60), one sample per pixel,
 * fused into one launch: initEyeRay, RayQuery_NearestHit, the resolve of
 * the preset's render_mode and Tonemap (MultiRenderer_resolve.cpp:536-542).
 * Render modes: LAMBERT_NO_TEX (ResolveCommon :580-666: white albedo, the
 * given lights), PHONG_NO_TEX (:668-732; its shadow ray is commented out
 * there), PBR_NO_TEX (:734-792, material 0), OUTLINE_PRIM (whose outline
 * test the reference applies only in OUTLINE_BORDER), GEOM, LOD, and with the scene's
 * COLORED materials (lrt_set_materials) LAMBERT, PHONG, PBR and DIFFUSE; and
 * kernel1D_ResolveDebug's
 * (:810-990) MASK, DEPTH, LINEAR_DEPTH, INVERSE_LINEAR_DEPTH, HSV_DEPTH,
 * PRIMITIVE, TYPE, MATERIAL, NORMAL, BARYCENTRIC, ST_ITERATIONS,
 * MO_VOXEL_COUNT and MO_FLAGS.  Misses take `background`.  The preset's
 * spp samples per pixel are traced through initEyeRay's sqrt(spp) grid (one
 * point for RAY_GEN_MODE_RANDOM), resolved with the sample-0 ray as
 * ResolveCommon does, and averaged; with a transparent COLORED material,
 * LAMBERT, PHONG, PBR and DIFFUSE take the reference's transparency path (the
 * AnyHit G-buffer blended into the resolved colour).  OUTLINE_BORDER
 * (ResolveOutline, :1073-1128) runs two launches per sample: a G-buffer pass
 * and the outline test against the four neighbours' t (more than 10 t / width
 * apart: colour (0.2, 0.2, 0.2)); it keeps 40 bytes per pixel of device
 * scratch with the scene.  TEXTURED materials (LAMBERT, PHONG, PBR, DIFFUSE;
 * PBR_NO_TEX's material 0) sample texture texId of lrt_set_textures at the
 * hit's texture coordinates, and TEX_COORDS shows those coordinates
 * (loadNormalTcFromGbuffer, :27-76: for triangles the barycentric blend of
 * the per-vertex coordinates of lrt_set_texcoords, zeros where none were set;
 * for SDF hits coords[0..1]).  Channel and intersection-count modes return
 * LRT_ERR_UNSUPPORTED; the pixel grid is the camera's (the reference pads
 * widths to a multiple of 8, and its outline test reads the padded grid).  Writes
 * width*height RGBA8 pixels (row-major) to device memory image_dev;
 * asynchronous on `stream`, lrt_trace_sync(stream) reports bounded-loop
 * limits.  No counterpart call in the reference (it renders through a
 * G-buffer); the node solver must be ST or BBOX. */
lrt_status lrt_render_rgba8(lrt_scene* scene, const lrt_camera* camera, const lrt_light* lights,
                            uint32_t light_count, const float background[4], uint32_t* image_dev, void* stream);

/* MultiRendererMaterial (core/IRenderer.h:31-38), 32 bytes. */
typedef struct lrt_material {
  uint32_t type; /* MULTI_RENDER_MATERIAL_TYPE_*, core/IRenderer.h:21-22 */
  uint32_t texId;
  float metallic;
  float roughness;
  float base_color[4];
} lrt_material;
enum { LRT_MATERIAL_COLORED = 0, LRT_MATERIAL_TEXTURED = 1 };

/* The renderer's materials (MultiRenderer::m_materials, m_matIdbyPrimId,
 * m_matIdOffsets: MultiRenderer.h:255-258), copied to the device: primitive
 * p of geometry g has material mat_id_by_prim_id[start_g + p % size_g] with
 * {start_g, size_g} = mat_id_offsets[2g .. 2g+1].  Every id must name a
 * material and every range lie inside mat_id_by_prim_id
 * (LRT_ERR_INVALID_ARGUMENT otherwise); a count of 0 clears them. */
lrt_status lrt_set_materials(lrt_scene* scene, const lrt_material* materials, uint32_t material_count,
                             const uint32_t* mat_id_by_prim_id, uint64_t mat_id_count, const uint32_t* mat_id_offsets,
                             uint32_t offset_count);

/* The renderer's textures (MultiRenderer::m_textures, MultiRenderer.h:256;
 * MultiRenderer::AddTexture, MultiRenderer_host.cpp:827-839): `count` float4
 * (RGBA) images, texture k of dims[2k] x dims[2k+1] texels (1..65536 each),
 * row-major, stored one after another in texels_rgba; every one is sampled
 * as the reference samples its textures, bilinear with clamped addressing
 * (Image2D<float4>::sample with Filter::LINEAR and AddressMode::CLAMP,
 * dependencies/1st-party/LiteMath/Image2d.cpp:50-183).  Texture k is what a
 * TEXTURED material with texId k samples (the reference renderer starts with
 * a 16x16 image of (0, 1, 1, 1) in every slot and AddTexture fills slots 1,
 * 2, ...: pass its slots as they are).  Copied to the device at the next
 * lrt_render_rgba8; a count of 0 clears them.  Texture coordinates beyond
 * +-2^31 / size convert differently (the reference's float-to-int
 * conversion of them is undefined). */
lrt_status lrt_set_textures(lrt_scene* scene, const float* texels_rgba, const uint32_t* dims, uint32_t count);

/* The per-vertex texture coordinates of triangle geometry geom_id (two
 * floats per vertex of its vertex array, in the order AddGeom_Triangles3f
 * received the vertices): what MultiRenderer::add_mesh_internal keeps in
 * m_vertices[].w / m_normals[].w (MultiRenderer_host.cpp:499-520) and the
 * resolve blends at a hit (loadNormalTcFromGbuffer, MultiRenderer_resolve.cpp:
 * 27-76).  vertex_count must equal the geometry's vertex count; 0 clears the
 * geometry's coordinates (they are then zero, as for a mesh loaded without
 * any). */
lrt_status lrt_set_texcoords(lrt_scene* scene, uint32_t geom_id, const float* texcoords, uint64_t vertex_count);

/* MultiRenderer::kernel1D_FillGbufferWithTransparency with AnyHit
 * (MultiRenderer.cpp:204-246), one sample of `camera`: per pixel the loop of
 * nearest hits that composites COLORED materials' base colours front to back
 * (misses take `background`; SBS_COL and graphics-primitive hits keep the
 * previous colour, as in the reference) until the remaining alpha is at most
 * 0.01, each ray restarting at the previous hit point.  Writes the float4
 * {rgb, alpha} to transparency_dev and the last hit to hits_dev (row-major
 * pixels, device memory); asynchronous on `stream`.  Every mesh geometry of
 * the scene needs a material range of size >= 1.  The reference's loop has
 * no bound; here a pixel stops after LRT_MAX_TRANSPARENCY_LAYERS traces and
 * lrt_trace_sync(stream) reports LRT_ERR_DEVICE_LIMIT. */
#define LRT_MAX_TRANSPARENCY_LAYERS 256
lrt_status lrt_fill_gbuffer_transparency(lrt_scene* scene, const lrt_camera* camera, const float background[4],
                                         float* transparency_dev, lrt_hit* hits_dev, void* stream);

/* Adjoint of lrt_render_lambert with respect to the scene's SBS float values
 * (the sdfSBSDataF array of the indexed layouts): grad_dev[j] +=
 * sum_i dimage_dev[i] * d image[i] / d values_f[j], by implicit
 * differentiation at each hit with the march recomputed (not stored).
 * grad_dev holds sdfSBSDataF_count floats and is accumulated into. */
lrt_status lrt_adjoint_lambert_sbs(lrt_scene* scene, const float* rays_dev, uint64_t n, const float light[3],
                                   const float* dimage_dev, float* grad_dev, void* stream);

/* lrt_adjoint_lambert_sbs over a width x height image of rays in 8x4-pixel
 * tiles and the stream's tile schedule, as lrt_render_lambert_image.  The
 * contributions are those of lrt_adjoint_lambert_sbs; only the order of the
 * float atomic additions into grad_dev differs. */
lrt_status lrt_adjoint_lambert_sbs_image(lrt_scene* scene, const float* rays_dev, uint32_t width, uint32_t height,
                                         const float light[3], const float* dimage_dev, float* grad_dev, void* stream,
                                         uint32_t flags);

/* Replaces the scene's SBS float values (count must equal the uploaded
 * sdfSBSDataF count; host memory, or device memory with
 * LRT_TRACE_DEVICE_POINTERS) and re-derives the device brick layouts. */
lrt_status lrt_sbs_update_values(lrt_scene* scene, const float* values_f, uint64_t count, void* stream,
                                 uint32_t flags);

/* ------------------------------------------------------------------------ */
/* Batched multi-camera form                                                */
/* ------------------------------------------------------------------------ */
/* The reference renders cameras one at a time (UpdateCamera + Render per
 * camera, render_CLI/offscreen_render.cpp:222-235).  A camera batch traces
 * the primary rays of many cameras of uneven sizes in ONE persistent launch:
 * each pixel's ray is generated in the kernel exactly as
 * lrt_generate_eye_rays does and traced exactly as lrt_trace_nearest does, so
 * every hit equals the per-camera path's.  The camera-table upload and the
 * launch are captured in a CUDA graph on first use and replayed afterwards.
 * Hits of camera i are at hits[offsets[i] + y*width + x]. */
typedef struct lrt_camera_batch lrt_camera_batch;

/* Launch shape: tiles of tile_w x tile_h pixels (tile_w * tile_h must be
 * 32 * rays_per_lane) taken by one warp at a time, each lane tracing
 * rays_per_lane pixels; stack_cap traversal-stack entries per thread in
 * shared memory (at least the scene's BLAS depth + 1, at most 81). */
typedef struct lrt_batch_shape {
  uint32_t tile_w;
  uint32_t tile_h;
  uint32_t rays_per_lane;
  uint32_t stack_cap;
} lrt_batch_shape;

typedef struct lrt_batch_tune_entry {
  lrt_batch_shape shape;
  float ms; /* mean time of one batched trace with this shape */
} lrt_batch_tune_entry;

#define LRT_BATCH_NO_GRAPH 0x1u /* lrt_batch_trace: launch directly instead of replaying the graph */

lrt_status lrt_batch_create(lrt_scene* scene, const lrt_camera* cams, uint32_t count, lrt_camera_batch** out);
lrt_status lrt_batch_destroy(lrt_camera_batch* batch);
/* count + 1 prefix offsets of the cameras' hits. */
lrt_status lrt_batch_ray_offsets(const lrt_camera_batch* batch, uint64_t* offsets);
/* New camera matrices (same image sizes); picked up by the next replay. */
lrt_status lrt_batch_update_cameras(lrt_camera_batch* batch, const lrt_camera* cams);
lrt_status lrt_batch_set_shape(lrt_camera_batch* batch, const lrt_batch_shape* shape);
lrt_status lrt_batch_get_shape(const lrt_camera_batch* batch, lrt_batch_shape* shape);
/* Asynchronous on `stream`; hits_dev: device memory for offsets[count] hits,
 * 16-byte aligned. */
lrt_status lrt_batch_trace(lrt_camera_batch* batch, lrt_hit* hits_dev, void* stream, uint32_t flags);
/* Waits for `stream`; LRT_ERR_DEVICE_LIMIT if a batched trace hit a bounded-loop limit. */
/* lrt_render_rgba8 for every camera of the batch in one launch (tiles and
 * launch shape of the batch): camera c's width*height RGBA8 pixels go to
 * images_dev + offsets[c] (lrt_batch_ray_offsets), row-major; every pixel
 * equals lrt_render_rgba8's for that camera.  Launched directly (no graph),
 * asynchronous on `stream`; lrt_batch_sync reports bounded-loop limits. */
lrt_status lrt_batch_render_rgba8(lrt_camera_batch* batch, const lrt_light* lights, uint32_t light_count,
                                  const float background[4], uint32_t* images_dev, void* stream);
lrt_status lrt_batch_sync(lrt_camera_batch* batch, void* stream);
/* The project autotuner: times every candidate shape (tiles 32x1, 16x2, 8x4,
 * 4x8 at 1 ray per lane, 16x4 and 8x8 at 2, 16x8 and 8x16 at 4; stack
 * capacities depth+1 and 81) over `reps` launches each on `stream`, keeps the
 * fastest, and reports every timing in `table` (up to table_cap entries). */
lrt_status lrt_batch_autotune(lrt_camera_batch* batch, lrt_hit* hits_dev, void* stream, uint32_t reps,
                              lrt_batch_tune_entry* table, uint32_t table_cap, uint32_t* table_len);

#ifdef __cplusplus
}
#endif
#endif /* LRT_B200_H */

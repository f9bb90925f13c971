// ref_harness.cpp — C entry points around the reference's own BVHRT.
//
// TEST INFRASTRUCTURE ONLY (oracle/_ref/liblrt_ref.so, the compiled-reference
// checker and CPU baseline).  Nothing here re-implements the ray query: every
// trace calls BVHRT::RayQuery_NearestHit (MultiRenderer/BVH2Common.cpp:
// 3322-3392) and every scene is assembled by the reference host code
// (AddGeom_* / AddInstance / CommitScene, MultiRenderer/BVH2Common_host.cpp)
// or by copying already-flattened arrays into the same BVHRT members.
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "MultiRenderer/BVH2Common.h"
#include "sdf/simple/sdf_simple.h"

#include "../../include/lrt_b200.h"
#include "abi_layout.h"
#include "ref_holder.h"

std::shared_ptr<ISceneObject> CreateSceneRT(const char* a_implName, const char* a_buildName, const char* a_layoutName);

namespace {
using Holder = LrtrHolder;

template <class T, class S>
void assign(std::vector<T>& dst, const S* src, uint64_t n)
{
  dst.resize(n);
  if (n) std::memcpy(dst.data(), src, n * sizeof(T));
}
} // namespace

extern "C" {

void* lrtr_create(const char* build_name, const char* layout_name)
{
  auto obj = CreateSceneRT("BVH2Common", build_name ? build_name : "cbvh_embree2",
                           layout_name ? layout_name : "SuperTreeletAlignedMerged4");
  if (!obj) return nullptr;
  Holder* h = new Holder{obj, dynamic_cast<BVHRT*>(obj->UnderlyingImpl(0))};
  h->rt->ClearGeom();
  return h;
}

void lrtr_destroy(void* p) { delete static_cast<Holder*>(p); }

void lrtr_set_preset(void* p, const lrt_preset* preset)
{
  MultiRenderPreset mp;
  std::memcpy(&mp, preset, sizeof(mp));
  static_cast<Holder*>(p)->rt->SetPreset(mp);
}

// getDefaultPreset() (core/render_settings.h:138-160) with sphere tracing and
// geometric normals: the preset the ray-query hot path is specified for.
void lrtr_set_parity_preset(void* p)
{
  MultiRenderPreset mp = getDefaultPreset();
  mp.sdf_node_intersect = SDF_OCTREE_NODE_INTERSECT_ST;
  mp.normal_mode = NORMAL_MODE_GEOMETRY;
  static_cast<Holder*>(p)->rt->SetPreset(mp);
}

uint32_t lrtr_add_triangles(void* p, const float* vpos3f, uint64_t nvert, const uint32_t* idx, uint64_t nidx)
{
  return static_cast<Holder*>(p)->rt->AddGeom_Triangles3f(vpos3f, nvert, idx, nidx, BUILD_HIGH, 12);
}

uint32_t lrtr_add_frame_octree(void* p, const lrt_sdf_frame_octree_node* nodes, uint64_t n)
{
  Holder* h = static_cast<Holder*>(p);
  SdfFrameOctreeView v;
  v.size = unsigned(n);
  v.nodes = reinterpret_cast<const SdfFrameOctreeNode*>(nodes);
  return h->rt->AddGeom_SdfFrameOctree(v, h->rt);
}

uint32_t lrtr_add_svs(void* p, const lrt_sdf_svs_node* nodes, uint64_t n)
{
  Holder* h = static_cast<Holder*>(p);
  SdfSVSView v;
  v.size = unsigned(n);
  v.nodes = reinterpret_cast<const SdfSVSNode*>(nodes);
  return h->rt->AddGeom_SdfSVS(v, h->rt);
}

uint32_t lrtr_add_sbs(void* p, const lrt_sdf_sbs_header* header, const lrt_sdf_sbs_node* nodes, uint64_t n,
                      const uint32_t* values, uint64_t nvalues, const float* values_f, uint64_t nvalues_f)
{
  Holder* h = static_cast<Holder*>(p);
  SdfSBSView v;
  std::memcpy(&v.header, header, sizeof(SdfSBSHeader));
  v.size = unsigned(n);
  v.nodes = reinterpret_cast<const SdfSBSNode*>(nodes);
  v.values_count = unsigned(nvalues);
  v.values = values;
  v.values_f_count = unsigned(nvalues_f);
  v.values_f = values_f;
  return h->rt->AddGeom_SdfSBS(v, h->rt);
}

uint32_t lrtr_add_instance(void* p, uint32_t geom_id, const float* m_col_major16)
{
  LiteMath::float4x4 m;
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) m(r, c) = m_col_major16[c * 4 + r];
  return static_cast<Holder*>(p)->rt->AddInstance(geom_id, m);
}

// BVHRT::UpdateInstance (BVH2Common_host.cpp:1303-1335) with the same matrix
// convention as lrtr_add_instance.
void lrtr_update_instance(void* p, uint32_t inst_id, const float* m_col_major16)
{
  LiteMath::float4x4 m;
  for (int c = 0; c < 4; c++)
    for (int r = 0; r < 4; r++) m(r, c) = m_col_major16[c * 4 + r];
  static_cast<Holder*>(p)->rt->UpdateInstance(inst_id, m);
}

void lrtr_commit(void* p) { static_cast<Holder*>(p)->rt->CommitScene(BUILD_HIGH); }

// View of the BVHRT members the traversal reads (BVH2Common.h:262-365).
void lrtr_export(void* p, lrt_scene_arrays* a)
{
  BVHRT* r = static_cast<Holder*>(p)->rt;
  std::memset(a, 0, sizeof(*a));
#define EXP(field, member, T)                                          \
  a->field = reinterpret_cast<T>(r->member.data());                      \
  a->field##_count = r->member.size();
  EXP(nodesTLAS, m_nodesTLAS, const lrt_bvh_node*)
  EXP(allNodePairs, m_allNodePairs, const lrt_bvh_node_pair*)
  EXP(instanceData, m_instanceData, const lrt_instance_data*)
  EXP(geomData, m_geomData, const lrt_geom_data*)
  EXP(geomTags, m_geomTags, const uint32_t*)
  EXP(startEnd, startEnd, const uint32_t*)
  EXP(primIdCount, m_primIdCount, const uint32_t*)
  EXP(indices, m_indices, const uint32_t*)
  EXP(vertPos, m_vertPos, const float*)
  EXP(primIndices, m_primIndices, const uint32_t*)
  EXP(origNodes, m_origNodes, const lrt_bvh_node*)
  EXP(sdfFrameOctreeNodes, m_SdfFrameOctreeNodes, const lrt_sdf_frame_octree_node*)
  EXP(sdfFrameOctreeRoots, m_SdfFrameOctreeRoots, const uint32_t*)
  EXP(sdfSVSNodes, m_SdfSVSNodes, const lrt_sdf_svs_node*)
  EXP(sdfSVSRoots, m_SdfSVSRoots, const uint32_t*)
  EXP(sdfSBSNodes, m_SdfSBSNodes, const lrt_sdf_sbs_node*)
  EXP(sdfSBSData, m_SdfSBSData, const uint32_t*)
  EXP(sdfSBSDataF, m_SdfSBSDataF, const float*)
  EXP(sdfSBSRoots, m_SdfSBSRoots, const uint32_t*)
  EXP(sdfSBSHeaders, m_SdfSBSHeaders, const lrt_sdf_sbs_header*)
#undef EXP
}

// Replace the BVHRT members with copies of already-flattened arrays.
void lrtr_import(void* p, const lrt_scene_arrays* a)
{
  BVHRT* r = static_cast<Holder*>(p)->rt;
  assign(r->m_nodesTLAS, a->nodesTLAS, a->nodesTLAS_count);
  assign(r->m_allNodePairs, a->allNodePairs, a->allNodePairs_count);
  assign(r->m_instanceData, a->instanceData, a->instanceData_count);
  assign(r->m_geomData, a->geomData, a->geomData_count);
  assign(r->m_geomTags, a->geomTags, a->geomTags_count);
  assign(r->startEnd, a->startEnd, a->startEnd_count);
  assign(r->m_primIdCount, a->primIdCount, a->primIdCount_count);
  assign(r->m_indices, a->indices, a->indices_count);
  assign(r->m_vertPos, a->vertPos, a->vertPos_count);
  assign(r->m_primIndices, a->primIndices, a->primIndices_count);
  assign(r->m_origNodes, a->origNodes, a->origNodes_count);
  assign(r->m_SdfFrameOctreeNodes, a->sdfFrameOctreeNodes, a->sdfFrameOctreeNodes_count);
  assign(r->m_SdfFrameOctreeRoots, a->sdfFrameOctreeRoots, a->sdfFrameOctreeRoots_count);
  assign(r->m_SdfSVSNodes, a->sdfSVSNodes, a->sdfSVSNodes_count);
  assign(r->m_SdfSVSRoots, a->sdfSVSRoots, a->sdfSVSRoots_count);
  assign(r->m_SdfSBSNodes, a->sdfSBSNodes, a->sdfSBSNodes_count);
  assign(r->m_SdfSBSData, a->sdfSBSData, a->sdfSBSData_count);
  assign(r->m_SdfSBSDataF, a->sdfSBSDataF, a->sdfSBSDataF_count);
  assign(r->m_SdfSBSRoots, a->sdfSBSRoots, a->sdfSBSRoots_count);
  assign(r->m_SdfSBSHeaders, a->sdfSBSHeaders, a->sdfSBSHeaders_count);
}

// n rays of {float4 posAndNear, float4 dirAndFar}; `threads` > 1 runs an
// OpenMP loop over rays (the reference ships the serial loop,
// MultiRenderer.cpp:187-190; RayQuery_NearestHit writes no members, so the
// parallel loop is race-free).
void lrtr_trace(void* p, const float* rays, lrt_hit* hits, uint64_t n, int threads)
{
  BVHRT* r = static_cast<Holder*>(p)->rt;
  if (threads <= 1) {
    for (uint64_t i = 0; i < n; i++) {
      const float* q = rays + 8 * i;
      CRT_Hit h = r->RayQuery_NearestHit(LiteMath::float4(q[0], q[1], q[2], q[3]),
                                         LiteMath::float4(q[4], q[5], q[6], q[7]));
      std::memcpy(&hits[i], &h, sizeof(h));
    }
    return;
  }
#pragma omp parallel for num_threads(threads) schedule(dynamic, 256)
  for (int64_t i = 0; i < int64_t(n); i++) {
    const float* q = rays + 8 * i;
    CRT_Hit h = r->RayQuery_NearestHit(LiteMath::float4(q[0], q[1], q[2], q[3]),
                                       LiteMath::float4(q[4], q[5], q[6], q[7]));
    std::memcpy(&hits[i], &h, sizeof(h));
  }
}

} // extern "C"

// bvhrt_b200.cpp — the reference-side drop-in of INTEGRATION.md, compiled:
// a BVHRT subclass that keeps the reference's own scene assembly and BVH
// build (AddGeom_*, AddInstance, CommitScene of MultiRenderer/
// BVH2Common_host.cpp) and hands the flattened members to liblrt_b200.so
// after every commit, so that ray queries run on the GPU.
//
// This is the file a LiteRT maintainer would add as
// MultiRenderer/BVH2Common_B200.cpp, plus one line in CreateSceneRT
// (BVH2Common_host.cpp:1594-1600):
//   if (std::string(a_implName) == "BVH2Common_B200")
//     return std::shared_ptr<ISceneObject>(new BVHRT_B200(a_buildName, a_layoutName));
// Here it is built against the reference's headers and objects into
// oracle/_ref/liblrt_b200_dropin.so (TEST INFRASTRUCTURE: the GPU tests drive
// it through the reference's own adders); lrtd_create stands in for that
// factory line, and ref_harness.cpp's lrtr_* entry points work on the result
// like on any BVHRT.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>

#include "MultiRenderer/BVH2Common.h"

#include "../../include/lrt_b200.h"
#include "abi_layout.h"
#include "ref_holder.h"

struct BVHRT_B200 : public BVHRT {
  lrt_scene* m_dev = nullptr;
  lrt_status m_status = LRT_OK;

  BVHRT_B200(const char* build, const char* layout) : BVHRT(build, layout) { lrt_scene_create(build, layout, &m_dev); }
  ~BVHRT_B200() override { lrt_scene_destroy(m_dev); }

  // the reference's TLAS build, then the reference's arrays to the device
  void CommitScene(uint32_t options) override
  {
    BVHRT::CommitScene(options);
    lrt_scene_arrays a;
    std::memset(&a, 0, sizeof(a));
#define LRTD_ARRAY(field, member)                              \
  a.field = reinterpret_cast<decltype(a.field)>(member.data()); \
  a.field##_count = member.size();
    LRTD_ARRAY(nodesTLAS, m_nodesTLAS)
    LRTD_ARRAY(allNodePairs, m_allNodePairs)
    LRTD_ARRAY(instanceData, m_instanceData)
    LRTD_ARRAY(geomData, m_geomData)
    LRTD_ARRAY(geomTags, m_geomTags)
    LRTD_ARRAY(startEnd, startEnd)
    LRTD_ARRAY(primIdCount, m_primIdCount)
    LRTD_ARRAY(indices, m_indices)
    LRTD_ARRAY(vertPos, m_vertPos)
    LRTD_ARRAY(primIndices, m_primIndices)
    LRTD_ARRAY(origNodes, m_origNodes)
    LRTD_ARRAY(sdfFrameOctreeNodes, m_SdfFrameOctreeNodes)
    LRTD_ARRAY(sdfFrameOctreeRoots, m_SdfFrameOctreeRoots)
    LRTD_ARRAY(sdfSVSNodes, m_SdfSVSNodes)
    LRTD_ARRAY(sdfSVSRoots, m_SdfSVSRoots)
    LRTD_ARRAY(sdfSBSNodes, m_SdfSBSNodes)
    LRTD_ARRAY(sdfSBSData, m_SdfSBSData)
    LRTD_ARRAY(sdfSBSDataF, m_SdfSBSDataF)
    LRTD_ARRAY(sdfSBSRoots, m_SdfSBSRoots)
    LRTD_ARRAY(sdfSBSHeaders, m_SdfSBSHeaders)
#undef LRTD_ARRAY
    lrt_preset p;
    std::memcpy(&p, &m_preset, sizeof(p)); // same layout, field by field (abi_layout.h)
    m_status = lrt_set_preset(m_dev, &p);
    if (m_status == LRT_OK) m_status = lrt_scene_upload(m_dev, &a);
    if (m_status != LRT_OK) std::fprintf(stderr, "BVHRT_B200::CommitScene: %s\n", lrt_last_error(m_dev));
  }

  // one ray: a 1-ray batch
  CRT_Hit RayQuery_NearestHit(LiteMath::float4 posAndNear, LiteMath::float4 dirAndFar) override
  {
    CRT_Hit h;
    lrt_ray_query_nearest_hit(m_dev, &posAndNear.x, &dirAndFar.x, reinterpret_cast<lrt_hit*>(&h));
    return h;
  }

  bool RayQuery_AnyHit(LiteMath::float4 posAndNear, LiteMath::float4 dirAndFar) override
  {
    int32_t r = 0;
    lrt_ray_query_any_hit(m_dev, &posAndNear.x, &dirAndFar.x, &r);
    return r != 0;
  }

  // what a B200 kernel1D_FillGbuffer calls: all rays of a frame at once
  lrt_status RayQuery_NearestHitBatch(const LiteMath::float4* rays, CRT_Hit* hits, uint64_t n)
  {
    return lrt_trace_nearest(m_dev, reinterpret_cast<const float*>(rays), reinterpret_cast<lrt_hit*>(hits), n,
                             nullptr, 0);
  }
};

extern "C" {

// CreateSceneRT("BVH2Common_B200", build, layout), wrapped like the
// checker's scenes (ref_holder.h) so that lrtr_* entry points accept it.
void* lrtd_create(const char* build_name, const char* layout_name)
{
  BVHRT_B200* rt = new BVHRT_B200(build_name ? build_name : "cbvh_embree2",
                                  layout_name ? layout_name : "SuperTreeletAlignedMerged4");
  if (!rt->m_dev) {
    delete rt;
    return nullptr;
  }
  LrtrHolder* h = new LrtrHolder{std::shared_ptr<ISceneObject>(rt), rt};
  h->rt->ClearGeom();
  return h;
}

// status of the last CommitScene's upload, and the library's message
int32_t lrtd_commit_status(void* p, char* msg, uint64_t cap)
{
  BVHRT_B200* rt = static_cast<BVHRT_B200*>(static_cast<LrtrHolder*>(p)->rt);
  if (msg && cap) std::snprintf(msg, cap, "%s", lrt_last_error(rt->m_dev));
  return int32_t(rt->m_status);
}

int32_t lrtd_trace_batch(void* p, const float* rays, lrt_hit* hits, uint64_t n)
{
  BVHRT_B200* rt = static_cast<BVHRT_B200*>(static_cast<LrtrHolder*>(p)->rt);
  return int32_t(rt->RayQuery_NearestHitBatch(reinterpret_cast<const LiteMath::float4*>(rays),
                                              reinterpret_cast<CRT_Hit*>(hits), n));
}

} // extern "C"

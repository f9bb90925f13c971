// render_harness.cpp — C entry points around the reference's own MultiRenderer.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle/_ref checker build).  A
// MultiRenderer (MultiRenderer/MultiRenderer*.cpp, compiled from the
// reference's sources) traces a scene held by ref_harness.cpp's BVHRT; this
// file only sets the renderer's state and calls its own code:
//   * initEyeRay (MultiRenderer.cpp:142-183) for the eye rays of an image,
//   * Render (MultiRenderer.cpp:14-60): kernel1D_FillGbuffer,
//     kernel1D_ResolveCommon / ResolveDebug / ResolveOutline,
//     kernel1D_FillGbufferWithTransparency + ResolveCommonWithTransparency,
//     kernel1D_Tonemap (MultiRenderer_resolve.cpp),
//   * kernel1D_FillGbufferWithTransparency with AnyHit (MultiRenderer.cpp:
//     204-246) alone, returning the transparency buffer and the G-buffer.
// The camera is given by its inverse matrices (the renderer's m_projInv and
// m_worldViewInv) or built by the reference's lookAt / perspectiveMatrix and
// UpdateCamera.  Image sizes must be multiples of 8: the renderer pads its
// tile grid to 8 and, for other sizes, writes past its G-buffer
// (kernel1D_FillGbuffer, MultiRenderer.cpp:190-200).
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "MultiRenderer/MultiRenderer.h"
#include "utils/mesh/mesh.h"

#include "../../include/lrt_b200.h"
#include "abi_layout.h"
#include "ref_holder.h"

namespace {

class HarnessRenderer : public MultiRenderer {
public:
  explicit HarnessRenderer(std::shared_ptr<ISceneObject> accel, BVHRT* rt) : MultiRenderer(AS_TYPE_COMMON), m_rt(rt)
  {
    SetAccelStruct(accel);
    m_preset = m_rt->m_preset;
  }

  void add_mesh(uint32_t geom_id, const float* v3, uint64_t nv, const uint32_t* idx, uint64_t ni, const float* tc2)
  {
    cmesh4::SimpleMesh m(nv, ni);
    for (uint64_t i = 0; i < nv; i++) {
      m.vPos4f[i] = LiteMath::float4(v3[3 * i], v3[3 * i + 1], v3[3 * i + 2], 1.0f);
      m.vNorm4f[i] = LiteMath::float4(0, 0, 0, 0);
      m.vTexCoord2f[i] = tc2 ? LiteMath::float2(tc2[2 * i], tc2[2 * i + 1]) : LiteMath::float2(0, 0);
    }
    for (uint64_t i = 0; i < ni; i++) m.indices[i] = idx[i];
    m.matIndices.clear();
    add_mesh_internal(m, geom_id);
  }

  void set_camera_inverse(const float* proj_inv, const float* world_view_inv)
  {
    for (int c = 0; c < 4; c++)
      for (int r = 0; r < 4; r++) {
        m_projInv(r, c) = proj_inv[c * 4 + r];
        m_worldViewInv(r, c) = world_view_inv[c * 4 + r];
      }
  }

  void set_materials(const lrt_material* mats, uint32_t n, const uint32_t* ids, uint64_t nids, const uint32_t* offs,
                     uint32_t ngeoms)
  {
    m_materials.resize(n);
    if (n) std::memcpy(m_materials.data(), mats, n * sizeof(lrt_material));
    m_matIdbyPrimId.assign(ids, ids + nids);
    m_matIdOffsets.resize(ngeoms);
    for (uint32_t g = 0; g < ngeoms; g++) m_matIdOffsets[g] = LiteMath::uint2(offs[2 * g], offs[2 * g + 1]);
    m_sceneHasLoadedMaterials = true;
  }

  // the instances' normal matrices, as MultiRenderer::AddInstance stores them
  void sync_instances()
  {
    m_instanceTransformInvTransposed.resize(m_rt->m_instanceData.size());
    for (size_t i = 0; i < m_rt->m_instanceData.size(); i++)
      m_instanceTransformInvTransposed[i] = m_rt->m_instanceData[i].transformInvTransposed;
  }

  void viewport(uint32_t w, uint32_t h)
  {
    SetViewport(0, 0, int(w), int(h));
    Clear(w, h);
  }

  void eye_rays(uint32_t w, uint32_t h, uint32_t sample, float* out)
  {
    viewport(w, h);
    for (uint32_t y = 0; y < h; y++)
      for (uint32_t x = 0; x < w; x++) {
        LiteMath::float4 p, d;
        initEyeRay(x, y, sample, &p, &d);
        float* o = out + 8 * (uint64_t(y) * w + x);
        std::memcpy(o, &p, 16);
        std::memcpy(o + 4, &d, 16);
      }
  }

  void render(uint32_t w, uint32_t h, uint32_t* image)
  {
    sync_instances();
    viewport(w, h);
    Render(image, w, h, 1);
  }

  void fill_transparency(uint32_t w, uint32_t h, uint32_t sample, float* transp, lrt_hit* gbuffer)
  {
    sync_instances();
    viewport(w, h);
    kernel1D_FillGbufferWithTransparency(m_packedXY_width * m_packedXY_height, sample);
    std::memcpy(transp, m_transparencyBuffer.data(), sizeof(float) * 4 * w * h);
    std::memcpy(gbuffer, m_gBuffer.data(), sizeof(lrt_hit) * w * h);
  }

  void set_frame(uint32_t frame) { m_AAFrameNum = frame; }

private:
  BVHRT* m_rt;
};

} // namespace

extern "C" {

void* lrtr_renderer_create(void* scene)
{
  LrtrHolder* h = static_cast<LrtrHolder*>(scene);
  return new HarnessRenderer(h->obj, h->rt);
}

void lrtr_renderer_destroy(void* r) { delete static_cast<HarnessRenderer*>(r); }

// add_mesh_internal's copy of a mesh; tc2: 2 texture coordinates per vertex (NULL: zeros)
void lrtr_renderer_add_mesh(void* r, uint32_t geom_id, const float* v3, uint64_t nv, const uint32_t* idx, uint64_t ni,
                            const float* tc2)
{
  static_cast<HarnessRenderer*>(r)->add_mesh(geom_id, v3, nv, idx, ni, tc2);
}

// MultiRenderer::AddTexture of a w x h float4 image (row-major); returns its slot
uint32_t lrtr_renderer_add_texture(void* r, uint32_t w, uint32_t h, const float* rgba)
{
  LiteImage::Image2D<LiteMath::float4> img(w, h, reinterpret_cast<const LiteMath::float4*>(rgba));
  return static_cast<HarnessRenderer*>(r)->AddTexture(img);
}

void lrtr_renderer_set_preset(void* r, const lrt_preset* p)
{
  MultiRenderPreset mp;
  std::memcpy(&mp, p, sizeof(mp));
  static_cast<HarnessRenderer*>(r)->SetPreset(mp);
}

void lrtr_renderer_set_camera_inverse(void* r, const float* proj_inv, const float* world_view_inv)
{
  static_cast<HarnessRenderer*>(r)->set_camera_inverse(proj_inv, world_view_inv);
}

// LiteMath lookAt / perspectiveMatrix (LiteMath.h:3315-3362) and
// MultiRenderer::UpdateCamera, which inverts both in float.
void lrtr_renderer_look_at(void* r, const float eye[3], const float center[3], const float up[3], float fovy,
                           float aspect, float znear, float zfar)
{
  const LiteMath::float4x4 view = LiteMath::lookAt(LiteMath::float3(eye[0], eye[1], eye[2]),
                                                   LiteMath::float3(center[0], center[1], center[2]),
                                                   LiteMath::float3(up[0], up[1], up[2]));
  const LiteMath::float4x4 proj = LiteMath::perspectiveMatrix(fovy, aspect, znear, zfar);
  static_cast<HarnessRenderer*>(r)->UpdateCamera(view, proj);
}

void lrtr_renderer_set_lights(void* r, const lrt_light* lights, uint32_t n)
{
  std::vector<Light> v(n);
  if (n) std::memcpy(v.data(), lights, n * sizeof(Light));
  static_cast<HarnessRenderer*>(r)->SetLights(v);
}

void lrtr_renderer_set_background(void* r, const float rgba[4])
{
  static_cast<HarnessRenderer*>(r)->setBackgroundColor(LiteMath::float4(rgba[0], rgba[1], rgba[2], rgba[3]));
}

void lrtr_renderer_set_materials(void* r, const lrt_material* mats, uint32_t n, const uint32_t* ids, uint64_t nids,
                                 const uint32_t* offsets, uint32_t ngeoms)
{
  static_cast<HarnessRenderer*>(r)->set_materials(mats, n, ids, nids, offsets, ngeoms);
}

void lrtr_renderer_set_frame(void* r, uint32_t frame) { static_cast<HarnessRenderer*>(r)->set_frame(frame); }

void lrtr_renderer_eye_rays(void* r, uint32_t w, uint32_t h, uint32_t sample, float* rays)
{
  static_cast<HarnessRenderer*>(r)->eye_rays(w, h, sample, rays);
}

void lrtr_renderer_render(void* r, uint32_t w, uint32_t h, uint32_t* image)
{
  static_cast<HarnessRenderer*>(r)->render(w, h, image);
}

void lrtr_renderer_fill_transparency(void* r, uint32_t w, uint32_t h, uint32_t sample, float* transp, lrt_hit* gbuffer)
{
  static_cast<HarnessRenderer*>(r)->fill_transparency(w, h, sample, transp, gbuffer);
}

} // extern "C"

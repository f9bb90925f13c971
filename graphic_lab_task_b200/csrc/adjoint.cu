// adjoint.cu — differentiable form of the SBS ray query (C-ABI lrt_render_lambert,
// lrt_adjoint_lambert_sbs, lrt_sbs_update_values).
//
// The reference has no differentiable renderer (its SparseDR sources are
// absent); this is the project's adjoint sphere tracer: the forward pass
// renders Lambert images through the same traversal as lrt_trace_nearest, the
// adjoint pass recomputes the march and scatters dLoss/d(SBS float values)
// by implicit differentiation at the hit (k_adjoint_lambert).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <iterator>
#include <cstring>

#include "device_scene.h"
#include "trace_api.h"

namespace lrt {
namespace {

// Re-resolves the dense corner grid and the surface-voxel mask of every brick
// of one indexed SBS model from the (new) float values.  One block per brick.
__global__ void k_sbs_rebuild(const lrt_sdf_sbs_node* __restrict__ nodes, const uint32_t* __restrict__ data,
                              const float* __restrict__ dataF, DevSbs sb, uint32_t root, float* __restrict__ dense,
                              uint32_t* __restrict__ mask)
{
  const uint32_t k = blockIdx.x;
  const uint32_t bs = sb.brick_size, V1 = bs + 1, P = sb.pad, V = sb.vsize;
  const uint32_t off = nodes[root + k].data_offset;
  float* g = dense + sb.denseBase + uint64_t(k) * sb.denseStride;
  for (uint32_t c = threadIdx.x; c < sb.denseStride; c += blockDim.x) {
    const uint32_t x = c / (V1 * V1), y = (c / V1) % V1, z = c % V1;
    g[c] = dataF[data[off + ((x + P) * V + (y + P)) * V + (z + P)]];
  }
  __syncthreads();
  uint32_t* m = mask + sb.maskBase + uint64_t(k) * sb.maskStride;
  for (uint32_t w = threadIdx.x; w < sb.maskStride; w += blockDim.x) m[w] = 0;
  __syncthreads();
  for (uint32_t v = threadIdx.x; v < bs * bs * bs; v += blockDim.x) {
    const uint32_t x = v / (bs * bs), y = (v / bs) % bs, z = v % bs;
    float vmin = 1e6f;
    for (int c = 0; c < 8; c++) {
      const float val = g[((x + ((c & 4) >> 2)) * V1 + (y + ((c & 2) >> 1))) * V1 + (z + (c & 1))];
      vmin = (val < vmin) ? val : vmin; // load_distance_values' reduction
    }
    if (vmin <= 0.0f) {
      atomicOr(m + 1 + v / 32, 1u << (v % 32));
      atomicOr(m, 1u);
    }
  }
}

lrt_status check_rays(lrt_scene* s, const void* p)
{
  if (!p || (reinterpret_cast<uintptr_t>(p) & 15))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "rays/outputs must be non-NULL 16-byte aligned device memory");
  return LRT_OK;
}

lrt_status begin(lrt_scene* s, cudaStream_t stream, StreamSlot** slot, DevScene* S)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->committed || !s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "render before CommitScene/upload");
  lrt_status st = check_preset(s, true);
  if (st != LRT_OK) return st;
  // a dedicated slot past the per-stream ones is not needed: render and
  // adjoint use the slot of their stream like lrt_trace_nearest
  DeviceScene* d = s->dev;
  auto it = d->slotOf.find(stream);
  int idx;
  if (it == d->slotOf.end()) {
    if (int(d->slotOf.size()) >= kMaxStreams)
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "more than %d streams used with one scene", kMaxStreams);
    idx = int(d->slotOf.size());
    d->slotOf[stream] = idx;
  } else {
    idx = it->second;
  }
  *slot = d->slots + idx;
  *S = d->S;
  S->flags = launch_flags(s);
  S->voxelStepCap = s->voxelStepCap ? s->voxelStepCap : kMaxVoxelSteps;
  cudaError_t e = cudaMemsetAsync(&(*slot)->work, 0, sizeof(unsigned long long), stream);
  return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "cudaMemsetAsync");
}

// The renderer's material tables on the device, copied when they changed
// since the last copy (synchronous: they change rarely).
lrt_status upload_materials(lrt_scene* s)
{
  DeviceScene* d = s->dev;
  if (d->matVersion == s->matVersion) return LRT_OK;
  cudaFree(d->mats);
  cudaFree(d->matIds);
  cudaFree(d->matOffsets);
  d->mats = nullptr;
  d->matIds = nullptr;
  d->matOffsets = nullptr;
  cudaError_t e = cudaMalloc(&d->mats, std::max<size_t>(1, s->mats.size()) * sizeof(lrt_material));
  if (e == cudaSuccess) e = cudaMalloc(&d->matIds, std::max<size_t>(1, s->matIds.size()) * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&d->matOffsets, std::max<size_t>(1, s->matOffsets.size()) * sizeof(uint32_t));
  if (e == cudaSuccess && !s->mats.empty())
    e = cudaMemcpy(d->mats, s->mats.data(), s->mats.size() * sizeof(lrt_material), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !s->matIds.empty())
    e = cudaMemcpy(d->matIds, s->matIds.data(), s->matIds.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !s->matOffsets.empty())
    e = cudaMemcpy(d->matOffsets, s->matOffsets.data(), s->matOffsets.size() * sizeof(uint32_t),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(s, e, "material tables host->device");
  d->matVersion = s->matVersion;
  return LRT_OK;
}

// Triangle slots of geometry g (its records in the triangle soup): one past
// the largest leaf range of its leaf table, as build_tri_soup counts them.
uint64_t triangle_slots(const HostArrays& h, size_t g)
{
  uint64_t ntri = 0;
  for (uint32_t a = h.startEnd[2 * g]; a < h.startEnd[2 * g + 1]; a++) {
    const uint32_t pk = h.primIdCount[a];
    ntri = std::max<uint64_t>(ntri, uint64_t(pk & 0x0FFFFFFFu) + ((pk & 0x70000000u) >> 28));
  }
  return ntri;
}

// Copies the textures and the triangles' texture coordinates to the device
// after they changed: the coordinates as 3 float2 per triangle slot (the
// triangle soup's indexing), zeros for geometries without coordinates.
lrt_status upload_textures(lrt_scene* s)
{
  DeviceScene* d = s->dev;
  if (d->texVersion == s->texVersion) return LRT_OK;
  cudaFree(d->texels);
  cudaFree(d->texTable);
  cudaFree(d->triTc);
  d->texels = nullptr;
  d->texTable = nullptr;
  d->triTc = nullptr;
  cudaError_t e = cudaSuccess;
  const size_t ntex = s->texDims.size() / 2;
  if (ntex) {
    std::vector<uint4> table(ntex);
    for (size_t k = 0; k < ntex; k++)
      table[k] = make_uint4(uint32_t(s->texOffsets[k]), s->texDims[2 * k], s->texDims[2 * k + 1], 0u);
    e = cudaMalloc(&d->texels, s->texels.size() * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&d->texTable, ntex * sizeof(uint4));
    if (e == cudaSuccess)
      e = cudaMemcpy(d->texels, s->texels.data(), s->texels.size() * sizeof(float), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d->texTable, table.data(), ntex * sizeof(uint4), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !s->texcoords.empty()) {
    const HostArrays& h = s->h;
    const size_t nslots = h.indices.size() / 3;
    std::vector<float> tc(std::max<size_t>(1, nslots) * 6, 0.0f);
    for (const auto& kv : s->texcoords) {
      const size_t g = kv.first;
      if (g >= h.geomData.size() || h.geomTags[g] != LRT_TAG_TRIANGLE) continue;
      const lrt_geom_data& gd = h.geomData[g];
      const uint64_t base = gd.offset[0] / 3, ntri = triangle_slots(h, g);
      for (uint64_t t = 0; t < ntri && base + t < nslots; t++)
        for (int c = 0; c < 3; c++) {
          const uint64_t vi = h.indices[gd.offset[0] + 3 * t + c];
          if (2 * vi + 1 < kv.second.size()) {
            tc[6 * (base + t) + 2 * c] = kv.second[2 * vi];
            tc[6 * (base + t) + 2 * c + 1] = kv.second[2 * vi + 1];
          }
        }
    }
    e = cudaMalloc(&d->triTc, tc.size() * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(d->triTc, tc.data(), tc.size() * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) return cuda_fail(s, e, "textures host->device");
  d->texVersion = s->texVersion;
  return LRT_OK;
}

// Every geometry whose hits read a material (all but the types in `skip`,
// a list ending in ~0u) needs a nonempty material range.
lrt_status check_material_ranges(lrt_scene* s, const char* who, const uint32_t* skip)
{
  const HostArrays& h = s->h;
  for (size_t g = 0; g < h.geomData.size(); g++) {
    const uint32_t type = h.geomData[g].type;
    bool skipped = false;
    for (const uint32_t* k = skip; *k != ~0u; k++) skipped |= type == *k;
    if (skipped) continue;
    if (2 * g + 1 >= s->matOffsets.size() || s->matOffsets[2 * g + 1] == 0)
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "%s: geometry %zu (type %u) has no material range (lrt_set_materials)",
                  who, g, type);
  }
  return LRT_OK;
}

// Shared arguments of the Lambert passes: width > 0 makes the n = width *
// height rays an image traced in 8x4-pixel tiles in the stream's tile
// schedule (natural tile order with LRT_TRACE_NATURAL_ORDER, the only flag).
lrt_status lambert_begin(lrt_scene* s, const char* who, const float* rays_dev, uint64_t n, uint32_t width,
                         uint32_t height, const float* light, uint32_t flags, cudaStream_t stream, StreamSlot** slot,
                         DevScene* S, int* grid)
{
  lrt_status st = begin(s, stream, slot, S);
  if (st != LRT_OK) return st;
  if (!light) return fail(s, LRT_ERR_INVALID_ARGUMENT, "%s: NULL light", who);
  if (flags & ~LRT_TRACE_NATURAL_ORDER) return fail(s, LRT_ERR_INVALID_ARGUMENT, "%s: unknown flags 0x%x", who, flags);
  if (width && (uint64_t(width / kImgTileW + 1) * (height / kImgTileH + 1) >= 0xFFFFFFFFull))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "%s: %u x %u pixels is more tiles than a launch can count", who, width,
                height);
  if ((st = check_rays(s, rays_dev)) != LRT_OK) return st;
  const uint64_t warps =
      width ? uint64_t((width + kImgTileW - 1) / kImgTileW) * ((height + kImgTileH - 1) / kImgTileH) : (n + 31) / 32;
  *grid = int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(s->dev->grid),
                                                       (warps * 32 + kTraceThreads - 1) / kTraceThreads)));
  return LRT_OK;
}

// A ray-order pass (width 0) of a wave or more of 32-ray groups that repeats
// the previous device trace's ray count on its stream (an optimisation loop's
// iterations) runs as an image 8 rays wide, whose 8x4 tiles are 32
// consecutive rays: the groups then follow the stream's schedule for that
// count, as lrt_trace_nearest's do.  Returns the image's width and height.
// Called once the call's arguments have been checked and its stream has a
// slot (the launch grid, a full wave, is the same in both shapes).
void rows_as_image(lrt_scene* s, cudaStream_t stream, uint64_t n, uint32_t flags, uint32_t& width, uint32_t& height)
{
  if (width) return;
  DeviceScene* d = s->dev;
  uint64_t& last = d->lastRays[stream];
  const bool repeat = last == n;
  last = n;
  const uint64_t slots = uint64_t(d->grid) * (kTraceThreads / 32);
  if (repeat && !(flags & LRT_TRACE_NATURAL_ORDER) && (n + 31) / 32 > slots && (n + 7) / 8 <= 0xFFFFFFFFull) {
    width = 8;
    height = uint32_t((n + 7) / 8);
  }
}

lrt_status render_lambert(lrt_scene* s, const float* rays_dev, uint64_t n, uint32_t width, uint32_t height,
                          const float light[3], float* image_dev, cudaStream_t stream, uint32_t flags)
{
  StreamSlot* slot = nullptr;
  DevScene S;
  int grid = 1;
  lrt_status st = lambert_begin(s, "lrt_render_lambert", rays_dev, n, width, height, light, flags, stream, &slot, &S,
                                &grid);
  if (st != LRT_OK) return st;
  if ((st = check_rays(s, image_dev)) != LRT_OK) return st;
  if (n == 0) return LRT_OK;
  rows_as_image(s, stream, n, flags, width, height);
  const bool natural = !width || (flags & LRT_TRACE_NATURAL_ORDER);
  const uint32_t* rd = nullptr;
  uint32_t* wr = nullptr;
  if ((st = sched_prepare(s, stream, width, height, natural, &rd, &wr)) != LRT_OK) return st;
  cudaError_t e = lrt_exact::launch_render_lambert(S, reinterpret_cast<const float4*>(rays_dev), n,
                                                   make_float3(light[0], light[1], light[2]), image_dev, &slot->work,
                                                   &slot->err, s->dev->stackCap, grid, stream, width, height, rd, wr);
  if (e != cudaSuccess) return cuda_fail(s, e, "render launch");
  sched_commit(s, stream, width, height, natural);
  return LRT_OK;
}

lrt_status adjoint_lambert(lrt_scene* s, const float* rays_dev, uint64_t n, uint32_t width, uint32_t height,
                           const float light[3], const float* dimage_dev, float* grad_dev, cudaStream_t stream,
                           uint32_t flags)
{
  StreamSlot* slot = nullptr;
  DevScene S;
  int grid = 1;
  lrt_status st = lambert_begin(s, "lrt_adjoint_lambert_sbs", rays_dev, n, width, height, light, flags, stream, &slot,
                                &S, &grid);
  if (st != LRT_OK) return st;
  if (!dimage_dev || !grad_dev) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_adjoint_lambert_sbs: NULL argument");
  if (n == 0) return LRT_OK;
  rows_as_image(s, stream, n, flags, width, height);
  const bool natural = !width || (flags & LRT_TRACE_NATURAL_ORDER);
  const uint32_t* rd = nullptr;
  uint32_t* wr = nullptr;
  if ((st = sched_prepare(s, stream, width, height, natural, &rd, &wr)) != LRT_OK) return st;
  cudaError_t e = lrt_exact::launch_adjoint_lambert(S, reinterpret_cast<const float4*>(rays_dev), n,
                                                    make_float3(light[0], light[1], light[2]), dimage_dev, grad_dev,
                                                    &slot->work, &slot->err, s->dev->stackCap, grid, stream, width,
                                                    height, rd, wr);
  if (e != cudaSuccess) return cuda_fail(s, e, "adjoint launch");
  sched_commit(s, stream, width, height, natural);
  return LRT_OK;
}

// OUTLINE_BORDER needs every pixel's neighbours' hits of the same sample: per
// sample a G-buffer pass (k_outline_fill, in the stream's tile schedule) and a
// resolve pass that applies the outline test and sums the samples; the last
// one tonemaps into the image.  The G-buffer (t and miss flag), the colours
// and the sums (8 + 16 + 16 bytes per pixel) are kept with the scene.
lrt_status render_outline_border(lrt_scene* s, const DevScene& S, StreamSlot* slot, const DevCamera& cam,
                                 const DevLights& L, const DevMaterials& M, const DevRenderModes& RM,
                                 uint32_t* image_dev, int grid, cudaStream_t stream)
{
  DeviceScene* d = s->dev;
  const uint64_t n = uint64_t(cam.width) * cam.height;
  auto up = [](uint64_t b) { return (b + 255) & ~uint64_t(255); };
  const uint64_t tmBytes = up(n * sizeof(float2)), colBytes = up(n * sizeof(float4));
  const uint64_t need = tmBytes + 2 * colBytes;
  cudaError_t e = cudaSuccess;
  if (need > d->outlineBytes) {
    if (d->outlineScratch) cudaFree(d->outlineScratch);
    d->outlineScratch = nullptr;
    d->outlineBytes = 0;
    if ((e = cudaMalloc(&d->outlineScratch, need)) != cudaSuccess) return cuda_fail(s, e, "outline G-buffer");
    d->outlineBytes = need;
  }
  char* base = static_cast<char*>(d->outlineScratch);
  float2* tm = reinterpret_cast<float2*>(base);
  float4* col = reinterpret_cast<float4*>(base + tmBytes);
  float4* acc = reinterpret_cast<float4*>(base + tmBytes + colBytes);
  for (uint32_t smp = 0; smp < RM.samples; smp++) {
    if (smp && (e = cudaMemsetAsync(&slot->work, 0, sizeof(unsigned long long), stream)) != cudaSuccess)
      return cuda_fail(s, e, "cudaMemsetAsync");
    const uint32_t* rd = nullptr;
    uint32_t* wr = nullptr;
    lrt_status st = sched_prepare(s, stream, cam.width, cam.height, false, &rd, &wr);
    if (st != LRT_OK) return st;
    e = lrt_exact::launch_outline_fill(S, cam, L, M, RM, smp, tm, col, &slot->work, &slot->err, d->stackCap, grid,
                                       stream, rd, wr);
    if (e != cudaSuccess) return cuda_fail(s, e, "outline G-buffer launch");
    sched_commit(s, stream, cam.width, cam.height, false);
    e = lrt_exact::launch_outline_resolve(tm, col, cam.width, cam.height, smp, RM.samples, acc, image_dev, stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "outline resolve launch");
  }
  return LRT_OK;
}

} // namespace
} // namespace lrt

using namespace lrt;

extern "C" {

lrt_status lrt_sbs_update_values(lrt_scene* s, const float* values_f, uint64_t count, void* stream_p,
                                 uint32_t flags)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->committed || !s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "lrt_sbs_update_values before upload");
  DeviceScene* d = s->dev;
  if (count != s->h.sdfSBSDataF.size() || !values_f)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_sbs_update_values: %llu values, the scene holds %zu",
                (unsigned long long)count, s->h.sdfSBSDataF.size());
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  float* dst = const_cast<float*>(d->S.sbsDataF);
  cudaError_t e = cudaMemcpyAsync(dst, values_f, count * sizeof(float),
                                  (flags & LRT_TRACE_DEVICE_POINTERS) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                  stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "lrt_sbs_update_values copy");
  // re-derive dense bricks and masks of the indexed models on the device
  for (size_t g = 0; g < s->h.geomData.size(); g++) {
    if (s->h.geomTags[g] != LRT_TAG_SDF_BRICK) continue;
    const uint32_t sid = s->h.geomData[g].offset[0];
    const DevSbs& sb = d->sbsHost[sid];
    if (!sb.colorLayout || sb.nodeCount == 0) continue;
    k_sbs_rebuild<<<sb.nodeCount, 128, 0, stream>>>(d->S.sbsNodes, d->S.sbsData, d->S.sbsDataF, sb,
                                                    s->h.sdfSBSRoots[sid], const_cast<float*>(d->S.sbsDense),
                                                    const_cast<uint32_t*>(d->S.sbsMask));
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(s, e, "brick rebuild");
  }
  // the pruned node pairs were derived from the old masks: trace the
  // unpruned pairs from now on
  d->S.pairs = d->pairsOrig;
  d->pfCand[1] = {d->pairsOrig, d->pairsOrigBytes}; // the node-pair entry of the prefetch ranges
  set_prefetch(d);
  return LRT_OK;
}

lrt_status lrt_render_rgba8(lrt_scene* s, const lrt_camera* camera, const lrt_light* lights, uint32_t light_count,
                            const float background[4], uint32_t* image_dev, void* stream_p)
{
  StreamSlot* slot = nullptr;
  DevScene S;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  lrt_status st = begin(s, stream, &slot, &S);
  if (st != LRT_OK) return st;
  if (!camera || !background || !image_dev || (light_count && !lights))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_render_rgba8: NULL camera, background, lights or image");
  if (light_count > LRT_MAX_LIGHTS)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_render_rgba8: %u lights (at most %d)", light_count, LRT_MAX_LIGHTS);
  const uint32_t mode = s->preset.render_mode;
  static const uint32_t kModes[] = {0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12,
                                    13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 24, 25};
  if (std::find(std::begin(kModes), std::end(kModes), mode) == std::end(kModes))
    return fail(s, LRT_ERR_UNSUPPORTED,
                "lrt_render_rgba8: render_mode %u (channels and intersection counts are outside the ray-query path)",
                mode);
  // a TEXTURED material samples texture texId (lrt_set_textures)
  auto material_ok = [&](const lrt_material& m) {
    return m.type == LRT_MATERIAL_COLORED || (m.type == LRT_MATERIAL_TEXTURED && m.texId < s->texDims.size() / 2);
  };
  if (mode == 11 && (s->mats.empty() || !material_ok(s->mats[0])))
    return fail(s, LRT_ERR_INVALID_ARGUMENT,
                "lrt_render_rgba8: PBR_NO_TEX shades with material 0, a COLORED one or a TEXTURED one whose texture "
                "is set");
  if (mode == 16 || mode == 17 || mode == 18 || mode == 21 || mode == 22) {
    // DIFFUSE, LAMBERT, PHONG and PBR read the materials; MATERIAL the material ids
    static const uint32_t kSkipDiffuse[] = {LRT_TYPE_SDF_SBS_COL, ~0u};
    static const uint32_t kSkipLambert[] = {LRT_TYPE_SDF_SBS_COL, LRT_TYPE_GRAPHICS_PRIM, ~0u};
    static const uint32_t kSkipNone[] = {~0u};
    st = check_material_ranges(s, "lrt_render_rgba8",
                               mode == 16 ? kSkipDiffuse : (mode == 21 || mode == 22) ? kSkipNone : kSkipLambert);
    if (st != LRT_OK) return st;
    if (mode != 22)
      for (size_t k = 0; k < s->mats.size(); k++)
        if (!material_ok(s->mats[k]))
          return fail(s, LRT_ERR_INVALID_ARGUMENT,
                      "lrt_render_rgba8: material %zu (type %u, texture %u of %zu set with lrt_set_textures)", k,
                      s->mats[k].type, s->mats[k].texId, s->texDims.size() / 2);
  }
  const uint32_t spp = s->preset.spp;
  if (spp == 0 || spp > 1024)
    return fail(s, LRT_ERR_UNSUPPORTED, "lrt_render_rgba8: spp %u (1..1024)", spp);
  DevRenderModes RM{};
  RM.mode = mode;
  RM.samples = spp;
  RM.sqrtSpp = uint32_t(std::sqrt(double(spp)));
  RM.invSqrt = 1.0f / float(RM.sqrtSpp);
  RM.random = s->preset.ray_gen_mode == 1; // RAY_GEN_MODE_RANDOM: the first Hamilton point
  RM.randomX = 0.5f;
  RM.randomY = float(0.333333);
  // CheckForTransparency (MultiRenderer.cpp:248-258): with a transparent
  // COLORED material, DIFFUSE, LAMBERT, PHONG and PBR go through the AnyHit
  // G-buffer and ResolveCommonWithTransparency (:33-46, :556-577)
  if (mode == 16 || mode == 17 || mode == 18 || mode == 21)
    for (const lrt_material& m : s->mats)
      if (m.type == LRT_MATERIAL_COLORED && m.base_color[3] < 1.0f) RM.transparency = 1;
  if (camera->width == 0 || camera->height == 0) return LRT_OK;
  if ((st = upload_materials(s)) != LRT_OK) return st;
  if ((st = upload_textures(s)) != LRT_OK) return st;
  DevCamera cam;
  std::memcpy(cam.proj_inv, camera->proj_inv, sizeof(cam.proj_inv));
  std::memcpy(cam.world_view_inv, camera->world_view_inv, sizeof(cam.world_view_inv));
  cam.width = camera->width;
  cam.height = camera->height;
  cam.tnear = camera->tnear;
  cam.tfar = camera->tfar;
  DevLights L{};
  if (light_count) std::memcpy(L.light, lights, light_count * sizeof(lrt_light));
  L.count = light_count;
  std::memcpy(L.background, background, sizeof(L.background));
  DeviceScene* d = s->dev;
  const uint64_t tiles = uint64_t((cam.width + 7) / 8) * ((cam.height + 3) / 4);
  const int grid = int(std::min<uint64_t>(uint64_t(d->grid), (tiles * 32 + kTraceThreads - 1) / kTraceThreads));
  const uint32_t* rd = nullptr;
  uint32_t* wr = nullptr;
  DevMaterials M{};
  M.mats = d->mats;
  M.ids = d->matIds;
  M.offsets = reinterpret_cast<const uint2*>(d->matOffsets);
  std::memcpy(M.background, background, sizeof(M.background));
  M.texels = d->texels;
  M.texs = d->texTable;
  M.texCount = d->texTable ? uint32_t(s->texDims.size() / 2) : 0u;
  M.triTc = d->triTc;
  if (mode == LRT_RENDER_MODE_OUTLINE_BORDER) return render_outline_border(s, S, slot, cam, L, M, RM, image_dev, grid, stream);
  if ((st = sched_prepare(s, stream, cam.width, cam.height, false, &rd, &wr)) != LRT_OK) return st;
  // one LAMBERT_NO_TEX sample of a brick-only scene: the 80-register kernel and its grid
  const bool bricks = d->bricksOnly && mode == LRT_RENDER_MODE_LAMBERT_NO_TEX && RM.samples == 1 && !RM.transparency;
  const int rgrid = bricks ? int(std::min<uint64_t>(uint64_t(d->gridBricks), (tiles * 32 + kTraceThreads - 1) / kTraceThreads))
                           : grid;
  const cudaError_t e = lrt_exact::launch_render_rgba8(S, cam, L, image_dev, &slot->work, &slot->err, d->stackCap,
                                                       rgrid, stream, rd, wr, &M, &RM, bricks);
  if (e != cudaSuccess) return cuda_fail(s, e, "render launch");
  sched_commit(s, stream, cam.width, cam.height, false);
  return LRT_OK;
}

lrt_status lrt_set_materials(lrt_scene* s, const lrt_material* materials, uint32_t material_count,
                             const uint32_t* mat_id_by_prim_id, uint64_t mat_id_count, const uint32_t* mat_id_offsets,
                             uint32_t offset_count)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if ((material_count && !materials) || (mat_id_count && !mat_id_by_prim_id) || (offset_count && !mat_id_offsets))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_materials: NULL array with a nonzero count");
  for (uint64_t i = 0; i < mat_id_count; i++)
    if (mat_id_by_prim_id[i] >= material_count)
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_materials: material id %u at %llu of %u materials",
                  mat_id_by_prim_id[i], (unsigned long long)i, material_count);
  for (uint32_t g = 0; g < offset_count; g++) {
    const uint64_t start = mat_id_offsets[2 * g], size = mat_id_offsets[2 * g + 1];
    if (start + size > mat_id_count)
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_materials: geometry %u range [%llu, +%llu) beyond %llu ids", g,
                  (unsigned long long)start, (unsigned long long)size, (unsigned long long)mat_id_count);
  }
  s->mats.assign(materials, materials + material_count);
  s->matIds.assign(mat_id_by_prim_id, mat_id_by_prim_id + mat_id_count);
  s->matOffsets.assign(mat_id_offsets, mat_id_offsets + 2 * size_t(offset_count));
  s->matVersion++;
  return LRT_OK;
}

lrt_status lrt_set_textures(lrt_scene* s, const float* texels_rgba, const uint32_t* dims, uint32_t count)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (count && (!texels_rgba || !dims))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_textures: NULL texels or sizes with %u textures", count);
  std::vector<uint64_t> offs(count);
  uint64_t total = 0;
  for (uint32_t k = 0; k < count; k++) {
    const uint64_t w = dims[2 * k], hgt = dims[2 * k + 1];
    if (w == 0 || hgt == 0 || w > (1u << 16) || hgt > (1u << 16))
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_textures: texture %u is %llu x %llu (1..65536 each way)", k,
                  (unsigned long long)w, (unsigned long long)hgt);
    offs[k] = total;
    total += w * hgt;
  }
  if (total >= (uint64_t(1) << 32))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_textures: %llu texels (fewer than 2^32)",
                (unsigned long long)total);
  s->texels.assign(texels_rgba, texels_rgba + 4 * total);
  s->texDims.assign(dims, dims + 2 * size_t(count));
  s->texOffsets = offs;
  s->texVersion++;
  return LRT_OK;
}

lrt_status lrt_set_texcoords(lrt_scene* s, uint32_t geom_id, const float* texcoords, uint64_t vertex_count)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  const HostArrays& h = s->h;
  if (geom_id >= h.geomData.size() || h.geomTags[geom_id] != LRT_TAG_TRIANGLE)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_texcoords: geometry %u is not a triangle mesh", geom_id);
  if (vertex_count == 0) {
    s->texcoords.erase(geom_id);
    s->texVersion++;
    return LRT_OK;
  }
  if (!texcoords) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_texcoords: NULL coordinates");
  // the geometry's vertices: from its vertex offset to the next mesh's (or the end)
  uint64_t end = h.vertPos.size() / 4;
  for (size_t g = 0; g < h.geomData.size(); g++)
    if (h.geomTags[g] == LRT_TAG_TRIANGLE && h.geomData[g].offset[1] > h.geomData[geom_id].offset[1])
      end = std::min<uint64_t>(end, h.geomData[g].offset[1]);
  const uint64_t nv = end - h.geomData[geom_id].offset[1];
  if (vertex_count != nv)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_set_texcoords: %llu coordinates for the %llu vertices of geometry %u",
                (unsigned long long)vertex_count, (unsigned long long)nv, geom_id);
  s->texcoords[geom_id].assign(texcoords, texcoords + 2 * vertex_count);
  s->texVersion++;
  return LRT_OK;
}

lrt_status lrt_fill_gbuffer_transparency(lrt_scene* s, const lrt_camera* camera, const float background[4],
                                         float* transparency_dev, lrt_hit* hits_dev, void* stream_p)
{
  StreamSlot* slot = nullptr;
  DevScene S;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  lrt_status st = begin(s, stream, &slot, &S);
  if (st != LRT_OK) return st;
  if (!camera || !background || !transparency_dev || !hits_dev)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_fill_gbuffer_transparency: NULL camera, background or output");
  if ((st = check_rays(s, transparency_dev)) != LRT_OK || (st = check_rays(s, hits_dev)) != LRT_OK) return st;
  static const uint32_t kSkip[] = {LRT_TYPE_SDF_SBS_COL, LRT_TYPE_GRAPHICS_PRIM, ~0u};
  if ((st = check_material_ranges(s, "lrt_fill_gbuffer_transparency", kSkip)) != LRT_OK) return st;
  if (camera->width == 0 || camera->height == 0) return LRT_OK;
  DeviceScene* d = s->dev;
  if ((st = upload_materials(s)) != LRT_OK) return st;
  DevCamera cam;
  std::memcpy(cam.proj_inv, camera->proj_inv, sizeof(cam.proj_inv));
  std::memcpy(cam.world_view_inv, camera->world_view_inv, sizeof(cam.world_view_inv));
  cam.width = camera->width;
  cam.height = camera->height;
  cam.tnear = camera->tnear;
  cam.tfar = camera->tfar;
  DevMaterials M;
  M.mats = d->mats;
  M.ids = d->matIds;
  M.offsets = reinterpret_cast<const uint2*>(d->matOffsets);
  std::memcpy(M.background, background, sizeof(M.background));
  const uint64_t tiles = uint64_t((cam.width + 7) / 8) * ((cam.height + 3) / 4);
  const int grid = int(std::min<uint64_t>(uint64_t(d->grid), (tiles * 32 + kTraceThreads - 1) / kTraceThreads));
  const uint32_t* rd = nullptr;
  uint32_t* wr = nullptr;
  if ((st = sched_prepare(s, stream, cam.width, cam.height, false, &rd, &wr)) != LRT_OK) return st;
  const cudaError_t e = lrt_exact::launch_fill_gbuffer_transparency(
      S, cam, M, reinterpret_cast<float4*>(transparency_dev), hits_dev, &slot->work, &slot->err, d->stackCap, grid,
      stream, rd, wr);
  if (e != cudaSuccess) return cuda_fail(s, e, "transparency launch");
  sched_commit(s, stream, cam.width, cam.height, false);
  return LRT_OK;
}

lrt_status lrt_render_lambert(lrt_scene* s, const float* rays_dev, uint64_t n, const float light[3], float* image_dev,
                              void* stream_p)
{
  return lrt::render_lambert(s, rays_dev, n, 0, 0, light, image_dev, static_cast<cudaStream_t>(stream_p), 0);
}

lrt_status lrt_render_lambert_image(lrt_scene* s, const float* rays_dev, uint32_t width, uint32_t height,
                                    const float light[3], float* image_dev, void* stream_p, uint32_t flags)
{
  return lrt::render_lambert(s, rays_dev, uint64_t(width) * height, width, height, light, image_dev,
                             static_cast<cudaStream_t>(stream_p), flags);
}

lrt_status lrt_adjoint_lambert_sbs(lrt_scene* s, const float* rays_dev, uint64_t n, const float light[3],
                                   const float* dimage_dev, float* grad_dev, void* stream_p)
{
  return lrt::adjoint_lambert(s, rays_dev, n, 0, 0, light, dimage_dev, grad_dev, static_cast<cudaStream_t>(stream_p),
                              0);
}

lrt_status lrt_adjoint_lambert_sbs_image(lrt_scene* s, const float* rays_dev, uint32_t width, uint32_t height,
                                         const float light[3], const float* dimage_dev, float* grad_dev,
                                         void* stream_p, uint32_t flags)
{
  return lrt::adjoint_lambert(s, rays_dev, uint64_t(width) * height, width, height, light, dimage_dev, grad_dev,
                              static_cast<cudaStream_t>(stream_p), flags);
}

} // extern "C"

// batch.cu — batched multi-camera form of the ray query (C-ABI in
// include/lrt_b200.h, lrt_batch_*).
//
// The reference renders cameras one after another: per camera UpdateCamera,
// then Render = initEyeRay + RayQuery_NearestHit per pixel
// (render_CLI/offscreen_render.cpp:222-235, MultiRenderer.cpp:142-202).  Here
// all cameras go through one persistent launch (k_trace_cameras) that
// generates each pixel's ray with the same function as lrt_generate_eye_rays
// and traces it with the same code as lrt_trace_nearest, so the hits equal
// the per-camera path's bit for bit.  The camera-table upload, the counter
// reset and the launch are captured once into a CUDA graph and replayed; an
// autotuner picks the launch shape (tile shape, rays per lane, stack size).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "device_scene.h"
#include "trace_api.h"

struct lrt_camera_batch {
  lrt_scene* scene = nullptr;
  uint32_t ncams = 0;
  std::vector<lrt_camera> cams;
  std::vector<uint64_t> offsets; // ncams + 1
  lrt::DevBatchShape shape{8, 4, 1, 0};
  uint32_t ntiles = 0;
  int grid = 0;
  // device / pinned state
  lrt::DevBatchCamera* hostTable = nullptr; // pinned, copied by the graph's memcpy node
  lrt::DevBatchCamera* devTable = nullptr;
  unsigned long long* state = nullptr; // [0] tile counter, [1] error word
  cudaStream_t capStream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  lrt_hit* graphHits = nullptr; // hits pointer baked into the graph
  lrt::DevScene graphScene{};   // scene parameters baked into the graph
  ~lrt_camera_batch()
  {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (capStream) cudaStreamDestroy(capStream);
    if (hostTable) cudaFreeHost(hostTable);
    if (devTable) cudaFree(devTable);
    if (state) cudaFree(state);
  }
};

namespace lrt {
namespace {

// Fills the pinned camera table for the current shape and returns the tile count.
void fill_table(lrt_camera_batch* b)
{
  uint32_t tile = 0;
  for (uint32_t i = 0; i < b->ncams; i++) {
    const lrt_camera& c = b->cams[i];
    DevBatchCamera& t = b->hostTable[i];
    std::memcpy(t.cam.proj_inv, c.proj_inv, sizeof(t.cam.proj_inv));
    std::memcpy(t.cam.world_view_inv, c.world_view_inv, sizeof(t.cam.world_view_inv));
    t.cam.width = c.width;
    t.cam.height = c.height;
    t.cam.tnear = c.tnear;
    t.cam.tfar = c.tfar;
    t.rayOffset = b->offsets[i];
    t.tilesX = (c.width + b->shape.tileW - 1) / b->shape.tileW;
    const uint32_t tilesY = (c.height + b->shape.tileH - 1) / b->shape.tileH;
    t.tileBase = tile;
    tile += t.tilesX * tilesY;
  }
  b->ntiles = tile;
}

lrt_status set_shape(lrt_camera_batch* b, const DevBatchShape& sh)
{
  lrt_scene* s = b->scene;
  if (sh.raysPerLane == 0 || sh.raysPerLane > 8 || sh.tileW == 0 || sh.tileW * sh.tileH != 32 * sh.raysPerLane)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "batch shape: tile_w * tile_h must equal 32 * rays_per_lane (1..8)");
  if (sh.stackCap < s->info.maxBlasDepth + 1 || sh.stackCap > kMaxStackDev + 1)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "batch shape: stack capacity %u outside [%u, %u]", sh.stackCap,
                s->info.maxBlasDepth + 1, kMaxStackDev + 1);
  int perSm = 0, sms = 0;
  cudaError_t e = lrt_exact::cameras_occupancy(sh.stackCap, &perSm);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  if (e != cudaSuccess) return cuda_fail(s, e, "batch occupancy");
  b->shape = sh;
  b->grid = std::max(1, perSm) * sms;
  fill_table(b);
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  return LRT_OK;
}

DevScene scene_params(lrt_scene* s)
{
  DevScene S = s->dev->S;
  S.flags = launch_flags(s);
  S.voxelStepCap = s->voxelStepCap ? s->voxelStepCap : kMaxVoxelSteps;
  return S;
}

// table upload + state reset + launch, on `stream` (captured or not); with
// `image`, RGBA8 pixels (resolve with `lights`) instead of hits
cudaError_t enqueue(lrt_camera_batch* b, lrt_hit* hits, cudaStream_t stream, const DevLights* lights = nullptr,
                    uint32_t* image = nullptr)
{
  cudaError_t e = cudaMemcpyAsync(b->devTable, b->hostTable, sizeof(DevBatchCamera) * b->ncams,
                                  cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->state, 0, sizeof(unsigned long long), stream);
  if (e == cudaSuccess) {
    const DevScene S = scene_params(b->scene);
    const int grid = int(std::min<uint64_t>(uint64_t(b->grid), (uint64_t(b->ntiles) * 32 + kTraceThreads - 1) / kTraceThreads));
    e = lrt_exact::launch_trace_cameras(S, b->devTable, b->ncams, b->ntiles, b->shape, hits, b->state,
                                        reinterpret_cast<uint32_t*>(b->state + 1), std::max(1, grid), stream, lights,
                                        image);
  }
  return e;
}

} // namespace
} // namespace lrt

using namespace lrt;

extern "C" {

lrt_status lrt_batch_create(lrt_scene* s, const lrt_camera* cams, uint32_t count, lrt_camera_batch** out)
{
  if (!s || !out) return LRT_ERR_INVALID_ARGUMENT;
  if (!cams || count == 0) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_batch_create: no cameras");
  if (!s->committed || !s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "lrt_batch_create before CommitScene/upload");
  lrt_status st = check_preset(s, true);
  if (st != LRT_OK) return st;
  lrt_camera_batch* b = new lrt_camera_batch();
  b->scene = s;
  b->ncams = count;
  b->cams.assign(cams, cams + count);
  b->offsets.resize(count + 1);
  b->offsets[0] = 0;
  for (uint32_t i = 0; i < count; i++) {
    if (cams[i].width == 0 || cams[i].height == 0 || cams[i].width > 65535 || cams[i].height > 65535) {
      delete b;
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_batch_create: camera %u has size %ux%u", i, cams[i].width,
                  cams[i].height);
    }
    b->offsets[i + 1] = b->offsets[i] + uint64_t(cams[i].width) * cams[i].height;
  }
  cudaError_t e = cudaMallocHost(&b->hostTable, sizeof(DevBatchCamera) * count);
  if (e == cudaSuccess) e = cudaMalloc(&b->devTable, sizeof(DevBatchCamera) * count);
  if (e == cudaSuccess) e = cudaMalloc(&b->state, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(b->state, 0, 2 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capStream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete b;
    return cuda_fail(s, e, "lrt_batch_create");
  }
  DevBatchShape sh{8, 4, 1, s->dev->stackCap};
  st = set_shape(b, sh);
  if (st != LRT_OK) {
    delete b;
    return st;
  }
  *out = b;
  return LRT_OK;
}

lrt_status lrt_batch_destroy(lrt_camera_batch* b)
{
  delete b;
  return LRT_OK;
}

lrt_status lrt_batch_ray_offsets(const lrt_camera_batch* b, uint64_t* offsets)
{
  if (!b || !offsets) return LRT_ERR_INVALID_ARGUMENT;
  std::memcpy(offsets, b->offsets.data(), sizeof(uint64_t) * b->offsets.size());
  return LRT_OK;
}

lrt_status lrt_batch_update_cameras(lrt_camera_batch* b, const lrt_camera* cams)
{
  if (!b || !cams) return LRT_ERR_INVALID_ARGUMENT;
  for (uint32_t i = 0; i < b->ncams; i++)
    if (cams[i].width != b->cams[i].width || cams[i].height != b->cams[i].height)
      return fail(b->scene, LRT_ERR_INVALID_ARGUMENT, "lrt_batch_update_cameras: camera %u changed size", i);
  b->cams.assign(cams, cams + b->ncams);
  fill_table(b); // the graph's memcpy node reads the pinned table at every replay
  return LRT_OK;
}

lrt_status lrt_batch_set_shape(lrt_camera_batch* b, const lrt_batch_shape* shape)
{
  if (!b || !shape) return LRT_ERR_INVALID_ARGUMENT;
  DevBatchShape sh{shape->tile_w, shape->tile_h, shape->rays_per_lane, shape->stack_cap};
  return set_shape(b, sh);
}

lrt_status lrt_batch_get_shape(const lrt_camera_batch* b, lrt_batch_shape* shape)
{
  if (!b || !shape) return LRT_ERR_INVALID_ARGUMENT;
  shape->tile_w = b->shape.tileW;
  shape->tile_h = b->shape.tileH;
  shape->rays_per_lane = b->shape.raysPerLane;
  shape->stack_cap = b->shape.stackCap;
  return LRT_OK;
}

lrt_status lrt_batch_trace(lrt_camera_batch* b, lrt_hit* hits_dev, void* stream_p, uint32_t flags)
{
  if (!b || !hits_dev) return LRT_ERR_INVALID_ARGUMENT;
  lrt_scene* s = b->scene;
  if (reinterpret_cast<uintptr_t>(hits_dev) & 15)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_batch_trace: hits must be 16-byte aligned");
  lrt_status st = check_preset(s, true);
  if (st != LRT_OK) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  cudaError_t e;
  if (flags & LRT_BATCH_NO_GRAPH) {
    e = enqueue(b, hits_dev, stream);
    return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "batched trace");
  }
  // re-capture when the hits buffer or anything the kernel reads from the
  // scene changed (preset, voxel limit, new SBS values, updated instances)
  const DevScene S = scene_params(s);
  if (!b->exec || b->graphHits != hits_dev || std::memcmp(&S, &b->graphScene, sizeof(S)) != 0) {
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    e = cudaStreamBeginCapture(b->capStream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(s, e, "cudaStreamBeginCapture");
    cudaError_t le = enqueue(b, hits_dev, b->capStream);
    e = cudaStreamEndCapture(b->capStream, &b->graph);
    if (le != cudaSuccess) return cuda_fail(s, le, "capturing the batched trace");
    if (e != cudaSuccess) return cuda_fail(s, e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) return cuda_fail(s, e, "cudaGraphInstantiate");
    b->graphHits = hits_dev;
    b->graphScene = S;
  }
  e = cudaGraphLaunch(b->exec, stream);
  return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "cudaGraphLaunch");
}

lrt_status lrt_batch_render_rgba8(lrt_camera_batch* b, const lrt_light* lights, uint32_t light_count,
                                  const float background[4], uint32_t* images_dev, void* stream_p)
{
  if (!b || !images_dev || !background || (light_count && !lights)) return LRT_ERR_INVALID_ARGUMENT;
  lrt_scene* s = b->scene;
  if (reinterpret_cast<uintptr_t>(images_dev) & 3)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_batch_render_rgba8: images must be 4-byte aligned");
  if (light_count > LRT_MAX_LIGHTS)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_batch_render_rgba8: %u lights (at most %d)", light_count,
                LRT_MAX_LIGHTS);
  if (s->preset.render_mode != LRT_RENDER_MODE_LAMBERT_NO_TEX)
    return fail(s, LRT_ERR_UNSUPPORTED, "lrt_batch_render_rgba8 renders the LAMBERT_NO_TEX mode (1), the preset has %u",
                s->preset.render_mode);
  lrt_status st = check_preset(s, true);
  if (st != LRT_OK) return st;
  DevLights L{};
  if (light_count) std::memcpy(L.light, lights, light_count * sizeof(lrt_light));
  L.count = light_count;
  std::memcpy(L.background, background, sizeof(L.background));
  const cudaError_t e = enqueue(b, nullptr, static_cast<cudaStream_t>(stream_p), &L, images_dev);
  return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "batched render");
}

lrt_status lrt_batch_sync(lrt_camera_batch* b, void* stream_p)
{
  if (!b) return LRT_ERR_INVALID_ARGUMENT;
  lrt_scene* s = b->scene;
  unsigned long long st[2];
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  cudaError_t e = cudaMemcpyAsync(st, b->state, sizeof(st), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "batched trace");
  const uint32_t err = uint32_t(st[1]);
  if (err) {
    cudaMemsetAsync(b->state + 1, 0, sizeof(unsigned long long), stream);
    cudaStreamSynchronize(stream);
    return fail(s, LRT_ERR_DEVICE_LIMIT, "batched trace hit a bounded-loop limit (error bits 0x%x)", err);
  }
  return LRT_OK;
}

// Times every candidate launch shape (reps launches each, CUDA events on
// `stream`) and keeps the fastest.  Candidates: tiles of 32x1, 16x2, 8x4,
// 4x8 (1 ray per lane), 16x4, 8x8 (2), 16x8, 8x16 (4); stack capacities of
// the scene's depth + 1 and the reference's 80 (+1).
lrt_status lrt_batch_autotune(lrt_camera_batch* b, lrt_hit* hits_dev, void* stream_p, uint32_t reps,
                              lrt_batch_tune_entry* table, uint32_t table_cap, uint32_t* table_len)
{
  if (!b || !hits_dev) return LRT_ERR_INVALID_ARGUMENT;
  lrt_scene* s = b->scene;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  if (reps == 0) reps = 3;
  const uint32_t need = s->info.maxBlasDepth + 1;
  const uint32_t tiles[8][3] = {{32, 1, 1}, {16, 2, 1}, {8, 4, 1}, {4, 8, 1}, {16, 4, 2}, {8, 8, 2}, {16, 8, 4}, {8, 16, 4}};
  std::vector<uint32_t> caps{std::max(need, 8u)};
  if (kMaxStackDev + 1 > caps[0]) caps.push_back(kMaxStackDev + 1);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  DevBatchShape bestShape = b->shape;
  uint32_t n = 0;
  lrt_status st = LRT_OK;
  for (const auto& t : tiles) {
    for (uint32_t cap : caps) {
      st = set_shape(b, DevBatchShape{t[0], t[1], t[2], cap});
      if (st != LRT_OK) break;
      cudaError_t e = enqueue(b, hits_dev, stream); // warm-up
      if (e == cudaSuccess) e = cudaEventRecord(e0, stream);
      for (uint32_t r = 0; r < reps && e == cudaSuccess; r++) e = enqueue(b, hits_dev, stream);
      if (e == cudaSuccess) e = cudaEventRecord(e1, stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(e1);
      float ms = 0;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
      if (e != cudaSuccess) {
        st = cuda_fail(s, e, "autotune");
        break;
      }
      ms /= float(reps);
      if (table && n < table_cap) table[n] = lrt_batch_tune_entry{{t[0], t[1], t[2], cap}, ms};
      n++;
      if (ms < best) {
        best = ms;
        bestShape = b->shape;
      }
    }
    if (st != LRT_OK) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (table_len) *table_len = n;
  if (st != LRT_OK) return st;
  st = set_shape(b, bestShape);
  if (st != LRT_OK) return st;
  return lrt_batch_sync(b, stream_p);
}

} // extern "C"

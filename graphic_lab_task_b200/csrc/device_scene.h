// device_scene.h — the device half of an lrt_scene (internal to liblrt_b200.so).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <tuple>
#include <vector>

#include "device_layout.h"
#include "scene.h"

namespace lrt {

// Per-stream launch state: the persistent grid's ray counter, the error word
// and the work counters.  One slot per stream keeps concurrent traces of one
// scene on different streams independent.
struct StreamSlot {
  unsigned long long work;
  unsigned long long counters[LRT_COUNTER_COUNT];
  uint32_t err;
  uint32_t _pad[5];
};
constexpr int kMaxStreams = 64;
// Host-pointer traces of at least kPipeMinRays rays run in chunks as a
// pipeline: host->device copies on one stream, device->host copies on
// another, and the traces round-robin over kPipeTraceStreams streams, so
// that both copy directions and the kernels of several chunks overlap.
constexpr int kPipeTraceStreams = 4;
constexpr int kPipeIn = 0, kPipeOut = 1, kPipeTrace = 2; // traces: kPipeTrace + k
constexpr int kPipeStreams = kPipeTrace + kPipeTraceStreams;
constexpr uint64_t kPipeChunk = 262144;   // 8 MiB of rays in, 8 MiB of hits out
constexpr uint64_t kPipeChunkMin = 32768; // first and last chunks
constexpr uint64_t kPipeMinRays = 262144;

// Tile schedule of the image-order launches of one image size on one stream
// (sched_next in trace_impl.cuh): two device buffers of sched_words(tiles)
// words, the one the next launch reads being buf[rd]; the other is cleared
// and written by that launch.  A scene keeps up to kMaxSchedules of them, so
// that launches alternating between image sizes on one stream keep their
// schedules (and allocate nothing after their first launch); beyond that
// the least recently used one is freed.
struct ImageSchedule {
  uint32_t* buf[2] = {nullptr, nullptr};
  int rd = 0;
  uint64_t lastUse = 0;
};
using SchedKey = std::tuple<cudaStream_t, uint32_t, uint32_t>; // stream, width, height
constexpr size_t kMaxSchedules = 32;

struct DeviceScene {
  std::vector<void*> allocs;
  DevScene S{};
  uint32_t stackCap = 0;
  int grid = 0;
  // every geometry is a sparse-brick set: image-order traces use the
  // 80-register kernel and its grid
  bool bricksOnly = false;
  int gridBricks = 0;
  StreamSlot* slots = nullptr; // device, kMaxStreams
  std::map<cudaStream_t, int> slotOf;
  const lrt_bvh_node_pair* pairsOrig = nullptr; // unpruned node pairs (used once SBS values change)
  uint64_t pairsOrigBytes = 0;
  // the arrays a trace may stream into L2 (DevScene::pfPtr), in priority
  // order, with their sizes; set_prefetch picks those that fit
  std::vector<std::pair<const void*, uint64_t>> pfCand;
  std::vector<DevSbs> sbsHost;                  // host copy of the SBS model table
  bool cleanBoxes = false;                      // every node box has 0 or 6 NaN coordinates
  bool pairsClean = false;                      // the BLAS part of cleanBoxes
  size_t tlasCount = 0, instCount = 0;          // sizes of the TLAS and instance buffers
  // per-tile hit counts of lrt_generate_bounce_rays_compact
  uint32_t* tileScratch = nullptr;
  uint64_t tileCap = 0;
  // keys, sorted keys, ray indices and radix-sort storage of
  // lrt_generate_bounce_rays_sorted
  void* sortScratch = nullptr;
  size_t sortBytes = 0;
  // G-buffer, colours and sums of the OUTLINE_BORDER render
  void* outlineScratch = nullptr;
  size_t outlineBytes = 0;
  // the renderer's material tables (lrt_set_materials), copied at the first
  // transparency trace after they changed
  lrt_material* mats = nullptr;
  uint32_t* matIds = nullptr;
  uint2* matOffsets = nullptr;
  uint64_t matVersion = 0;
  // the renderer's textures and the triangles' texture coordinates
  // (lrt_set_textures / lrt_set_texcoords), copied at the next render after they changed
  float4* texels = nullptr;
  uint4* texTable = nullptr;
  float2* triTc = nullptr;
  uint64_t texVersion = 0;
  std::map<SchedKey, ImageSchedule> sched; // per stream and image size of image-order launches
  uint64_t schedUses = 0;
  // ray count of the last device-pointer lrt_trace_nearest on each stream: a
  // trace of the same count again has its 32-ray groups scheduled
  std::map<cudaStream_t, uint64_t> lastRays;
  // staging buffers for host-pointer calls
  float4* rays = nullptr;
  lrt_hit* hits = nullptr;
  uint64_t cap = 0;
  // streams of the chunked host-pointer pipeline (created on first use);
  // pipeEv[p] orders stream p's chunk before the next stage, pipeStart the
  // pipeline after the work already queued on the caller's stream
  cudaStream_t pipe[kPipeStreams] = {};
  cudaEvent_t pipeEv[kPipeStreams] = {};
  cudaEvent_t pipeStart = nullptr;
  uint32_t* pipeErrHost = nullptr; // page-locked copy of the pipeline's error word
  // device address of lrt_trace_nearest_noalloc's static scratch array on
  // this scene's device, looked up at upload (and the lookup's result)
  unsigned char* noallocBase = nullptr;
  cudaError_t noallocErr = cudaSuccess;
  ~DeviceScene()
  {
    if (pipeErrHost) cudaFreeHost(pipeErrHost);
    for (int p = 0; p < kPipeStreams; p++) {
      if (pipe[p]) cudaStreamDestroy(pipe[p]);
      if (pipeEv[p]) cudaEventDestroy(pipeEv[p]);
    }
    if (pipeStart) cudaEventDestroy(pipeStart);
    for (void* p : allocs) cudaFree(p);
    if (rays) cudaFree(rays);
    if (hits) cudaFree(hits);
    if (tileScratch) cudaFree(tileScratch);
    if (sortScratch) cudaFree(sortScratch);
    if (outlineScratch) cudaFree(outlineScratch);
    if (mats) cudaFree(mats);
    if (matIds) cudaFree(matIds);
    if (matOffsets) cudaFree(matOffsets);
    if (texels) cudaFree(texels);
    if (texTable) cudaFree(texTable);
    if (triTc) cudaFree(triTc);
    for (auto& kv : sched)
      for (uint32_t* b : kv.second.buf) cudaFree(b);
  }
};

// device.cu
uint32_t preset_flags(const lrt_preset& p);
// The schedule buffers of the next image-order launch of a width x height
// image on `stream` (allocated on the first launch of that size on that
// stream); *rd = *wr = nullptr when `natural` asks for plain tile order.
// The caller launches, then calls sched_commit with the same arguments.
lrt_status sched_prepare(lrt_scene* s, cudaStream_t stream, uint32_t width, uint32_t height, bool natural,
                         const uint32_t** rd, uint32_t** wr);
void sched_commit(lrt_scene* s, cudaStream_t stream, uint32_t width, uint32_t height, bool natural);
uint32_t launch_flags(const lrt_scene* s); // preset flags + the uploaded scene's own
// DevScene::pfPtr/pfBytes from d->pfCand: the candidates in order while
// their sum stays within kPrefetchMaxBytes
void set_prefetch(DeviceScene* d);
lrt_status cuda_fail(lrt_scene* s, cudaError_t e, const char* what);

} // namespace lrt

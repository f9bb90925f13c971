// device.cu — device half of the scene object: upload of the reference arrays
// plus the derived layouts, and the ray-query entry points of the C-ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "device_scene.h"
#include "layout.h"
#include "scene.h"
#include "trace_api.h"

namespace lrt {

lrt_status cuda_fail(lrt_scene* s, cudaError_t e, const char* what)
{
  return fail(s, e == cudaErrorMemoryAllocation ? LRT_ERR_OUT_OF_MEMORY : LRT_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
}

uint32_t preset_flags(const lrt_preset& p)
{
  const uint32_t m = p.render_mode; // need_normal(), BVH2Common.cpp:19-32
  const bool nn = m == 1 || m == 8 || m == 12 || m == 17 || m == 20 || m == 7 || m == 18 || m == 23 || m == 21 ||
                  m == 11 || m == 27;
  uint32_t f = 0;
  if (nn) f |= kFlagNeedNormal;
  if (m == LRT_RENDER_MODE_ST_ITERATIONS) f |= kFlagStIterations;
  if (p.representation_mode == 0) f |= kFlagSurfaceMode;
  if (p.sdf_node_intersect == 3) f |= kFlagBBoxMode;
  f |= (p.sdf_node_intersect & 7u) << kFlagSolverShift;
  return f;
}

uint32_t launch_flags(const lrt_scene* s)
{
  return preset_flags(s->preset) | (s->dev->cleanBoxes ? kFlagCleanBoxes : 0u);
}

namespace {

// True if every box of the nodes has either no NaN coordinate or six.
bool boxes_clean(const lrt_bvh_node* n, size_t count)
{
  for (size_t i = 0; i < count; i++) {
    int nans = 0;
    for (int k = 0; k < 3; k++) nans += std::isnan(n[i].boxMin[k]) + std::isnan(n[i].boxMax[k]);
    if (nans != 0 && nans != 6) return false;
  }
  return true;
}

template <class T>
lrt_status upload_vec(lrt_scene* s, DeviceScene* d, const T* src, size_t count, const T** out, const char* name)
{
  *out = nullptr;
  if (count == 0) return LRT_OK;
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, count * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(s, e, name);
  d->allocs.push_back(p);
  e = cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(s, e, name);
  *out = static_cast<const T*>(p);
  return LRT_OK;
}

lrt_status slot_for(lrt_scene* s, cudaStream_t stream, StreamSlot** out)
{
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
  *out = d->slots + idx;
  return LRT_OK;
}

} // namespace

lrt_status sched_prepare(lrt_scene* s, cudaStream_t stream, uint32_t width, uint32_t height, bool natural,
                         const uint32_t** rd, uint32_t** wr)
{
  *rd = nullptr;
  *wr = nullptr;
  if (natural) return LRT_OK;
  DeviceScene* d = s->dev;
  const uint64_t tiles = uint64_t((width + kImgTileW - 1) / kImgTileW) * ((height + kImgTileH - 1) / kImgTileH);
  const size_t clear = sched_lists_offset(tiles) * sizeof(uint32_t); // header, bitmap, cost accumulators
  cudaError_t e = cudaSuccess;
  const SchedKey key(stream, width, height);
  auto it = d->sched.find(key);
  if (it == d->sched.end()) {
    if (d->sched.size() >= kMaxSchedules) { // free the least recently used schedule
      auto old = d->sched.begin();
      for (auto jt = d->sched.begin(); jt != d->sched.end(); ++jt)
        if (jt->second.lastUse < old->second.lastUse) old = jt;
      for (uint32_t* b : old->second.buf) cudaFree(b);
      d->sched.erase(old);
    }
    ImageSchedule fresh;
    for (uint32_t*& b : fresh.buf) {
      if (e == cudaSuccess) e = cudaMalloc(&b, sched_words(tiles) * sizeof(uint32_t));
      if (e == cudaSuccess) e = cudaMemsetAsync(b, 0, clear, stream);
    }
    if (e != cudaSuccess) {
      for (uint32_t* b : fresh.buf) cudaFree(b);
      return cuda_fail(s, e, "tile schedule buffers");
    }
    it = d->sched.emplace(key, fresh).first;
  }
  ImageSchedule& q = it->second;
  q.lastUse = ++d->schedUses;
  e = cudaMemsetAsync(q.buf[1 - q.rd], 0, clear, stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaMemsetAsync");
  *rd = q.buf[q.rd];
  *wr = q.buf[1 - q.rd];
  return LRT_OK;
}

void sched_commit(lrt_scene* s, cudaStream_t stream, uint32_t width, uint32_t height, bool natural)
{
  if (natural) return;
  auto it = s->dev->sched.find(SchedKey(stream, width, height));
  if (it != s->dev->sched.end()) it->second.rd = 1 - it->second.rd;
}

namespace {

// img_w > 0: the n = img_w * img_h rays are an image in row-major order,
// traced in 8x4-pixel tiles, in the stream's tile schedule unless flags has
// LRT_TRACE_NATURAL_ORDER (or LRT_TRACE_COUNT_WORK).
// err: the error word the kernel reports into (default: the slot's).
lrt_status launch(lrt_scene* s, const float4* rays, lrt_hit* hits, uint64_t n, cudaStream_t stream, uint32_t flags,
                  StreamSlot* slot, uint32_t img_w = 0, uint32_t img_h = 0, uint32_t* err = nullptr)
{
  if (!err) err = &slot->err;
  DeviceScene* d = s->dev;
  DevScene S = d->S;
  S.flags = launch_flags(s);
  S.voxelStepCap = s->voxelStepCap ? s->voxelStepCap : kMaxVoxelSteps;
  if (n < kPrefetchMinRays)
    for (int r = 0; r < kPrefetchRanges; r++) S.pfBytes[r] = 0;
  const bool count = (flags & LRT_TRACE_COUNT_WORK) != 0;
  cudaError_t e = cudaMemsetAsync(&slot->work, 0, count ? offsetof(StreamSlot, err) : sizeof(unsigned long long),
                                  stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaMemsetAsync");
  // Row order: rays to a warp.  A launch of fewer rays than one wave of the
  // kernel's warps can hold takes as long as its slowest warp, and a warp's
  // time grows with the number of slow rays among its lanes, so such a launch
  // gives each warp 16 or 8 rays while the warps still fit in one wave, taken
  // with a stride across the launch's rays (k_trace).
  uint32_t group = 32;
  if (!img_w) {
    const uint64_t slots = uint64_t(d->grid) * (kTraceThreads / 32);
    while (group > 8 && (n + group / 2 - 1) / (group / 2) <= slots) group /= 2;
  }
  const uint64_t warps = img_w ? uint64_t((img_w + kImgTileW - 1) / kImgTileW) * ((img_h + kImgTileH - 1) / kImgTileH)
                               : (n + group - 1) / group;
  // image-order traces of brick-only scenes use the 80-register kernel (its own grid)
  const bool bricks = img_w && !count && d->bricksOnly;
  const int grid = int(std::min<uint64_t>(uint64_t(bricks ? d->gridBricks : d->grid),
                                          (warps * 32 + kTraceThreads - 1) / kTraceThreads));
  const bool natural = !img_w || count || (flags & LRT_TRACE_NATURAL_ORDER);
  const uint32_t* rd = nullptr;
  uint32_t* wr = nullptr;
  lrt_status st = sched_prepare(s, stream, img_w, img_h, natural, &rd, &wr);
  if (st != LRT_OK) return st;
  if (flags & LRT_TRACE_FAST_MATH)
    e = lrt_fast::launch_trace(S, rays, hits, n, &slot->work, slot->counters, err, d->stackCap, grid, stream, count,
                               img_w, img_h, rd, wr, group, bricks);
  else
    e = lrt_exact::launch_trace(S, rays, hits, n, &slot->work, slot->counters, err, d->stackCap, grid, stream,
                                count, img_w, img_h, rd, wr, group, bricks);
  if (e != cudaSuccess) return cuda_fail(s, e, "trace launch");
  sched_commit(s, stream, img_w, img_h, natural);
  return LRT_OK;
}

lrt_status limit_fail(lrt_scene* s, uint32_t bits)
{
  return fail(s, LRT_ERR_DEVICE_LIMIT,
              "trace hit a bounded-loop limit (error bits 0x%x: 1 = stack, 2 = voxel march, 4 = transparency layers)",
              bits);
}

// Reads back (and clears) the error word and, if asked, the counters of a slot.
lrt_status finish(lrt_scene* s, cudaStream_t stream, StreamSlot* slot, bool count)
{
  StreamSlot hs;
  cudaError_t e = cudaMemcpyAsync(&hs, slot, sizeof(hs), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "trace");
  if (count)
    for (int k = 0; k < LRT_COUNTER_COUNT; k++) s->counters[k] = hs.counters[k];
  if (hs.err) {
    cudaMemsetAsync(&slot->err, 0, sizeof(uint32_t), stream);
    cudaStreamSynchronize(stream);
    return limit_fail(s, hs.err);
  }
  return LRT_OK;
}

// Chunk sizes of the pipeline: kPipeChunkMin, doubling up to kPipeChunk,
// chunks of at most kPipeChunk, and the ramp again in reverse, so that the
// first copy in and the last trace and copy out, which nothing overlaps, are
// short.  Inputs too small for the ramps get chunks of kPipeChunkMin.
void pipeline_chunks(uint64_t n, std::vector<uint64_t>& out)
{
  out.clear();
  std::vector<uint64_t> up;
  uint64_t ramp = 0;
  for (uint64_t m = kPipeChunkMin; m < kPipeChunk; m *= 2) {
    up.push_back(m);
    ramp += m;
  }
  if (n <= 2 * ramp) {
    for (uint64_t off = 0; off < n; off += kPipeChunkMin) out.push_back(std::min(kPipeChunkMin, n - off));
    return;
  }
  out = up;
  const uint64_t mid = n - 2 * ramp;
  const uint64_t parts = (mid + kPipeChunk - 1) / kPipeChunk;
  for (uint64_t i = 0; i < parts; i++) out.push_back(mid / parts + (i < mid % parts ? 1 : 0));
  out.insert(out.end(), up.rbegin(), up.rend());
}

// Host-pointer trace in chunks (staging buffers already hold n rays): chunk c
// is copied in on kPipeIn, traced on trace stream c mod kPipeTraceStreams
// once its copy is done, and copied out on kPipeOut once its trace is done.
// The copies of consecutive chunks run back to back in both directions while
// the traces of several chunks run at the same time.  The pipeline starts
// after the work already queued on the caller's stream, and the caller's
// stream waits for it.  Events are re-recorded once per chunk: a wait takes
// the record made before it.  Every trace reports into one error word, which
// the copy-out stream (that has waited for every trace) reads into page-locked
// host memory after the last hits, so one synchronisation ends the call.
lrt_status trace_host_pipelined(lrt_scene* s, const float* rays, lrt_hit* hits, uint64_t n, cudaStream_t stream,
                                uint32_t flags)
{
  DeviceScene* d = s->dev;
  cudaError_t e = cudaSuccess;
  if (!d->pipeStart) {
    for (int p = 0; p < kPipeStreams && e == cudaSuccess; p++) {
      e = cudaStreamCreateWithFlags(&d->pipe[p], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d->pipeEv[p], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaHostAlloc(&d->pipeErrHost, sizeof(uint32_t), cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d->pipeStart, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(s, e, "pipeline streams");
  }
  cudaStream_t in = d->pipe[kPipeIn], out = d->pipe[kPipeOut];
  StreamSlot* slots[kPipeTraceStreams];
  for (int k = 0; k < kPipeTraceStreams; k++) {
    lrt_status st = slot_for(s, d->pipe[kPipeTrace + k], &slots[k]);
    if (st != LRT_OK) return st;
  }
  uint32_t* err = &slots[0]->err;
  e = cudaEventRecord(d->pipeStart, stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(in, d->pipeStart, 0);
  if (e != cudaSuccess) return cuda_fail(s, e, "pipeline start");
  lrt_status st = LRT_OK;
  std::vector<uint64_t> chunks;
  pipeline_chunks(n, chunks);
  for (uint64_t off = 0, c = 0; c < chunks.size(); off += chunks[c], c++) {
    const uint64_t m = chunks[c];
    const int k = int(c % kPipeTraceStreams);
    cudaStream_t tr = d->pipe[kPipeTrace + k];
    e = cudaMemcpyAsync(d->rays + 2 * off, rays + 8 * off, m * 32, cudaMemcpyHostToDevice, in);
    if (e == cudaSuccess) e = cudaEventRecord(d->pipeEv[kPipeIn], in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(tr, d->pipeEv[kPipeIn], 0);
    if (e != cudaSuccess) {
      st = cuda_fail(s, e, "rays host->device");
      break;
    }
    st = launch(s, d->rays + 2 * off, d->hits + off, m, tr, flags, slots[k], 0, 0, err);
    if (st != LRT_OK) break;
    e = cudaEventRecord(d->pipeEv[kPipeTrace + k], tr);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(out, d->pipeEv[kPipeTrace + k], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(hits + off, d->hits + off, m * sizeof(lrt_hit), cudaMemcpyDeviceToHost, out);
    if (e != cudaSuccess) {
      st = cuda_fail(s, e, "hits device->host");
      break;
    }
  }
  if (st == LRT_OK) {
    e = cudaMemcpyAsync(d->pipeErrHost, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, out);
    if (e != cudaSuccess) st = cuda_fail(s, e, "error word");
  }
  // the caller's stream waits for the last copy out
  if (cudaEventRecord(d->pipeEv[kPipeOut], out) == cudaSuccess) cudaStreamWaitEvent(stream, d->pipeEv[kPipeOut], 0);
  if (st != LRT_OK) { // drain every stream after a failure
    for (int p = 0; p < kPipeStreams; p++) cudaStreamSynchronize(d->pipe[p]);
    cudaMemsetAsync(err, 0, sizeof(uint32_t), out);
    cudaStreamSynchronize(out);
    return st;
  }
  e = cudaStreamSynchronize(out);
  if (e != cudaSuccess) return cuda_fail(s, e, "hits device->host");
  const uint32_t bits = *d->pipeErrHost;
  if (bits) {
    cudaMemsetAsync(err, 0, sizeof(uint32_t), out);
    cudaStreamSynchronize(out);
    return limit_fail(s, bits);
  }
  return LRT_OK;
}

} // namespace

// Device address of the static scratch array of lrt_trace_nearest_noalloc
// (defined with it at the end of this file), for the current device.
cudaError_t noalloc_scratch_address(void** p);

lrt_status device_upload(lrt_scene* s)
{
  device_release(s);
  cudaError_t e = cudaGetDevice(&s->device);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaGetDevice (no CUDA device?)");
  DeviceScene* d = new DeviceScene();
  s->dev = d;
  const HostArrays& h = s->h;
  DevScene& S = d->S;
  std::vector<DevGeom> geoms;
  std::vector<float> soup, dense;
  std::vector<DevSbs> sbs;
  std::vector<uint32_t> mask;
  build_geoms(h, geoms);
  build_tri_soup(h, soup);
  build_sbs_dense(h, sbs, dense);
  build_sbs_masks(h, sbs, dense, mask);
  std::vector<lrt_bvh_node_pair> pairs;
  prune_sbs_pairs(h, geoms, sbs, mask, pairs);
  lrt_status st = LRT_OK;
#define UP(dst, vec, T, name)                                                                        \
  if (st == LRT_OK) {                                                                                 \
    const T* p = nullptr;                                                                             \
    st = upload_vec(s, d, reinterpret_cast<const T*>(vec.data()), vec.size() * sizeof(vec[0]) / sizeof(T), &p, name); \
    S.dst = p;                                                                                        \
  }
  UP(tlas, h.nodesTLAS, lrt_bvh_node, "TLAS nodes")
  UP(pairs, pairs, lrt_bvh_node_pair, "BLAS node pairs")
  UP(instances, h.instanceData, DevInstance, "instances")
  UP(geoms, geoms, DevGeom, "geometry table")
  UP(primIdCount, h.primIdCount, uint32_t, "leaf table")
  UP(triSoup, soup, float4, "triangles")
  UP(primIndices, h.primIndices, uint32_t, "primIndices")
  UP(origNodes, h.origNodes, lrt_bvh_node, "origNodes")
  UP(frameOctreeNodes, h.sdfFrameOctreeNodes, lrt_sdf_frame_octree_node, "frame-octree nodes")
  UP(svsNodes, h.sdfSVSNodes, lrt_sdf_svs_node, "SVS nodes")
  UP(sbsNodes, h.sdfSBSNodes, lrt_sdf_sbs_node, "SBS nodes")
  UP(sbsData, h.sdfSBSData, uint32_t, "SBS data")
  UP(sbsDataF, h.sdfSBSDataF, float, "SBS float data")
  UP(sbsDense, dense, float, "SBS dense bricks")
  UP(sbsMask, mask, uint32_t, "SBS surface-voxel masks")
  UP(sbs, sbs, DevSbs, "SBS table")
  if (st == LRT_OK) {
    if (h.sdfSBSNodes.empty()) {
      d->pairsOrig = S.pairs; // nothing was pruned
    } else {
      const lrt_bvh_node_pair* p = nullptr;
      st = upload_vec(s, d, h.allNodePairs.data(), h.allNodePairs.size(), &p, "unpruned node pairs");
      d->pairsOrig = p;
    }
  }
  d->sbsHost = sbs;
  d->pairsOrigBytes = (h.sdfSBSNodes.empty() ? pairs.size() : h.allNodePairs.size()) * sizeof(lrt_bvh_node_pair);
  // what a traversal reads per node, leaf, brick and voxel, most shared first
  d->pfCand = {{S.tlas, h.nodesTLAS.size() * sizeof(lrt_bvh_node)},
               {S.pairs, pairs.size() * sizeof(lrt_bvh_node_pair)},
               {S.primIdCount, h.primIdCount.size() * sizeof(uint32_t)},
               {S.sbsNodes, h.sdfSBSNodes.size() * sizeof(lrt_sdf_sbs_node)},
               {S.sbsMask, mask.size() * sizeof(uint32_t)},
               {S.triSoup, soup.size() * sizeof(float)},
               {S.origNodes, h.origNodes.size() * sizeof(lrt_bvh_node)},
               {S.frameOctreeNodes, h.sdfFrameOctreeNodes.size() * sizeof(lrt_sdf_frame_octree_node)},
               {S.svsNodes, h.sdfSVSNodes.size() * sizeof(lrt_sdf_svs_node)},
               {S.sbsDense, dense.size() * sizeof(float)}};
  set_prefetch(d);
  d->pairsClean = boxes_clean(reinterpret_cast<const lrt_bvh_node*>(pairs.data()), 2 * pairs.size()) &&
                  boxes_clean(reinterpret_cast<const lrt_bvh_node*>(h.allNodePairs.data()), 2 * h.allNodePairs.size());
  d->cleanBoxes = d->pairsClean && boxes_clean(h.nodesTLAS.data(), h.nodesTLAS.size());
  d->tlasCount = h.nodesTLAS.size();
  d->instCount = h.instanceData.size();
#undef UP
  if (st != LRT_OK) {
    device_release(s);
    return st;
  }
  d->stackCap = std::max<uint32_t>(s->info.maxBlasDepth + 1, 8u);
  // The dynamic shared-memory limit is a per-kernel attribute shared by all
  // scenes: raise it once to the largest stack any scene may use.
  e = lrt_exact::set_trace_smem(kMaxStack + 1);
  if (e == cudaSuccess) e = lrt_fast::set_trace_smem(kMaxStack + 1);
  int perSm = 0, perSmBricks = 0, sms = 0;
  d->bricksOnly = !h.geomTags.empty() &&
                  std::all_of(h.geomTags.begin(), h.geomTags.end(), [](uint32_t t) { return t == LRT_TAG_SDF_BRICK; });
  if (e == cudaSuccess) e = lrt_exact::trace_occupancy(d->stackCap, &perSm);
  if (e == cudaSuccess) e = lrt_exact::trace_occupancy(d->stackCap, &perSmBricks, true);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
  if (e == cudaSuccess) e = cudaMalloc(&d->slots, sizeof(StreamSlot) * kMaxStreams);
  if (e == cudaSuccess) {
    d->allocs.push_back(d->slots);
    e = cudaMemset(d->slots, 0, sizeof(StreamSlot) * kMaxStreams);
  }
  if (e != cudaSuccess) {
    st = cuda_fail(s, e, "trace setup");
    device_release(s);
    return st;
  }
  d->grid = std::max(1, perSm) * sms;
  d->gridBricks = std::max(1, perSmBricks) * sms;
  // The allocation-free trace's static array is looked up here, with the
  // scene's device current, not in the trace call: under lazy module loading
  // the first lookup loads this file's module and places the array in device
  // memory, which an upload may do and lrt_trace_nearest_noalloc must not.
  // A failed lookup fails only that entry point.
  void* base = nullptr;
  d->noallocErr = noalloc_scratch_address(&base);
  if (d->noallocErr != cudaSuccess) cudaGetLastError(); // not sticky: clear it
  d->noallocBase = static_cast<unsigned char*>(base);
  return LRT_OK;
}

// After a commit that changed only instances (UpdateInstance, or ClearScene
// and AddInstance over the same geometry): write the new TLAS and instances
// into their buffers (new buffers where the counts changed) and leave every
// BLAS, brick and mask array on the device as it is.
lrt_status device_update_instances(lrt_scene* s)
{
  DeviceScene* d = s->dev;
  const HostArrays& h = s->h;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev != s->device)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "commit on device %d of a scene uploaded to device %d", dev, s->device);
  lrt_status st = LRT_OK;
  auto put = [&](const void* src, size_t count, size_t elem, size_t& have, const void** ptr, const char* name) {
    if (st != LRT_OK) return;
    if (count != have) {
      void* p = nullptr;
      e = cudaMalloc(&p, count * elem);
      if (e != cudaSuccess) {
        st = cuda_fail(s, e, name);
        return;
      }
      d->allocs.push_back(p);
      *ptr = p; // the old buffer stays listed in allocs and is freed with the scene
      have = count;
    }
    e = cudaMemcpy(const_cast<void*>(*ptr), src, count * elem, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_fail(s, e, name);
  };
  put(h.nodesTLAS.data(), h.nodesTLAS.size(), sizeof(lrt_bvh_node), d->tlasCount,
      reinterpret_cast<const void**>(&d->S.tlas), "TLAS nodes");
  put(h.instanceData.data(), h.instanceData.size(), sizeof(lrt_instance_data), d->instCount,
      reinterpret_cast<const void**>(&d->S.instances), "instances");
  if (st != LRT_OK) return st;
  d->cleanBoxes = d->pairsClean && boxes_clean(h.nodesTLAS.data(), h.nodesTLAS.size());
  return LRT_OK;
}

void set_prefetch(DeviceScene* d)
{
  DevScene& S = d->S;
  uint64_t total = 0;
  int k = 0;
  for (int r = 0; r < kPrefetchRanges; r++) {
    S.pfPtr[r] = nullptr;
    S.pfBytes[r] = 0;
  }
  for (const auto& c : d->pfCand) {
    const uint64_t bytes = c.second & ~uint64_t(15); // whole 16-byte granules (cudaMalloc bases are aligned)
    if (!c.first || bytes == 0 || k == kPrefetchRanges || total + bytes > kPrefetchMaxBytes) continue;
    S.pfPtr[k] = static_cast<const char*>(c.first);
    S.pfBytes[k] = bytes;
    total += bytes;
    k++;
  }
}

void device_release(lrt_scene* s)
{
  if (s->dev) {
    delete s->dev;
    s->dev = nullptr;
  }
}

} // namespace lrt

using namespace lrt;

extern "C" {

lrt_status lrt_trace_nearest(lrt_scene* s, const float* rays, lrt_hit* hits, uint64_t n, void* stream_p,
                             uint32_t flags)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->committed || !s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "trace before CommitScene/upload");
  if (n == 0) return LRT_OK;
  if (!rays || !hits) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_trace_nearest: NULL rays or hits");
  lrt_status st = check_preset(s);
  if (st != LRT_OK) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  StreamSlot* slot = nullptr;
  st = slot_for(s, stream, &slot);
  if (st != LRT_OK) return st;
  DeviceScene* d = s->dev;
  if (flags & LRT_TRACE_DEVICE_POINTERS) {
    if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15)
      return fail(s, LRT_ERR_INVALID_ARGUMENT, "device rays/hits must be 16-byte aligned");
    // A trace of a wave or more of 32-ray groups that repeats the previous
    // trace's ray count on this stream (a renderer's frames) goes through the
    // image-order kernel as an image 8 rays wide, whose 8x4 tiles are the same
    // 32 consecutive rays: the groups are then handed out in the stream's
    // schedule for this ray count (slowest groups first, the slowest split
    // over two warps when the previous launch was tail-bound).  Traces of
    // changing counts keep plain row order and allocate no schedule.
    uint64_t& last = d->lastRays[stream];
    const bool repeat = last == n;
    last = n;
    const uint64_t slots = uint64_t(d->grid) * (kTraceThreads / 32);
    if (repeat && !(flags & (LRT_TRACE_COUNT_WORK | LRT_TRACE_NATURAL_ORDER)) && (n + 15) / 16 > slots &&
        (n + 7) / 8 <= 0xFFFFFFFFull)
      return launch(s, reinterpret_cast<const float4*>(rays), hits, n, stream, flags, slot, 8, uint32_t((n + 7) / 8));
    return launch(s, reinterpret_cast<const float4*>(rays), hits, n, stream, flags, slot);
  }
  if (n > d->cap) {
    if (d->rays) cudaFree(d->rays);
    if (d->hits) cudaFree(d->hits);
    d->rays = nullptr;
    d->hits = nullptr;
    d->cap = 0;
    cudaError_t e = cudaMalloc(&d->rays, n * 32);
    if (e == cudaSuccess) e = cudaMalloc(&d->hits, n * sizeof(lrt_hit));
    if (e != cudaSuccess) return cuda_fail(s, e, "staging buffers");
    d->cap = n;
  }
  if (n >= kPipeMinRays && !(flags & LRT_TRACE_COUNT_WORK)) return trace_host_pipelined(s, rays, hits, n, stream, flags);
  cudaError_t e = cudaMemcpyAsync(d->rays, rays, n * 32, cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "rays host->device");
  st = launch(s, d->rays, d->hits, n, stream, flags, slot);
  if (st != LRT_OK) return st;
  e = cudaMemcpyAsync(hits, d->hits, n * sizeof(lrt_hit), cudaMemcpyDeviceToHost, stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "hits device->host");
  return finish(s, stream, slot, (flags & LRT_TRACE_COUNT_WORK) != 0);
}

lrt_status lrt_trace_nearest_image(lrt_scene* s, const float* rays_dev, lrt_hit* hits_dev, uint32_t width,
                                   uint32_t height, void* stream_p, uint32_t flags)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->committed || !s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "trace before CommitScene/upload");
  if (width == 0 || height == 0) return LRT_OK;
  if (!rays_dev || !hits_dev || ((reinterpret_cast<uintptr_t>(rays_dev) | reinterpret_cast<uintptr_t>(hits_dev)) & 15))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_trace_nearest_image: rays/hits must be 16-byte aligned device memory");
  lrt_status st = check_preset(s);
  if (st != LRT_OK) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  StreamSlot* slot = nullptr;
  st = slot_for(s, stream, &slot);
  if (st != LRT_OK) return st;
  return launch(s, reinterpret_cast<const float4*>(rays_dev), hits_dev, uint64_t(width) * height, stream, flags, slot,
                width, height);
}

// Waits for the stream's traces and reports a bounded-loop limit hit by any of
// them (device-pointer traces are asynchronous).
lrt_status lrt_trace_sync(lrt_scene* s, void* stream_p, int32_t read_counters)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "no device scene");
  StreamSlot* slot = nullptr;
  lrt_status st = slot_for(s, static_cast<cudaStream_t>(stream_p), &slot);
  if (st != LRT_OK) return st;
  return finish(s, static_cast<cudaStream_t>(stream_p), slot, read_counters != 0);
}

lrt_status lrt_ray_query_nearest_hit(lrt_scene* s, const float pn[4], const float df[4], lrt_hit* out)
{
  if (!s || !pn || !df || !out) return fail(s, LRT_ERR_INVALID_ARGUMENT, "RayQuery_NearestHit: NULL argument");
  float ray[8];
  std::memcpy(ray, pn, 16);
  std::memcpy(ray + 4, df, 16);
  return lrt_trace_nearest(s, ray, out, 1, nullptr, 0);
}

lrt_status lrt_ray_query_any_hit(lrt_scene* s, const float pn[4], const float df[4], int32_t* out)
{
  if (!s || !pn || !df || !out) return fail(s, LRT_ERR_INVALID_ARGUMENT, "RayQuery_AnyHit: NULL argument");
  // BVH2Common.cpp:3394-3399: negate tfar to request stop-on-first-hit
  float d2[4] = {df[0], df[1], df[2], -df[3]};
  lrt_hit h;
  lrt_status st = lrt_ray_query_nearest_hit(s, pn, d2, &h);
  if (st != LRT_OK) return st;
  *out = h.geomId != 0xFFFFFFFFu;
  return LRT_OK;
}

lrt_status lrt_set_voxel_step_limit(lrt_scene* s, uint32_t steps)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  s->voxelStepCap = steps;
  return LRT_OK;
}

lrt_status lrt_get_work_counters(lrt_scene* s, uint64_t counters[LRT_COUNTER_COUNT])
{
  if (!s || !counters) return LRT_ERR_INVALID_ARGUMENT;
  std::memcpy(counters, s->counters, sizeof(s->counters));
  return LRT_OK;
}

lrt_status lrt_generate_eye_rays(lrt_scene* s, const lrt_camera* cam, float* rays_dev, void* stream)
{
  if (!cam || !rays_dev) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_generate_eye_rays: NULL argument");
  if (reinterpret_cast<uintptr_t>(rays_dev) & 15)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "rays must be 16-byte aligned");
  DevCamera c;
  std::memcpy(c.proj_inv, cam->proj_inv, sizeof(c.proj_inv));
  std::memcpy(c.world_view_inv, cam->world_view_inv, sizeof(c.world_view_inv));
  c.width = cam->width;
  c.height = cam->height;
  c.tnear = cam->tnear;
  c.tfar = cam->tfar;
  cudaError_t e = lrt_exact::launch_eye_rays(c, reinterpret_cast<float4*>(rays_dev), static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return s ? cuda_fail(s, e, "eye rays") : LRT_ERR_CUDA;
  return LRT_OK;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free trace (lrt_trace_nearest_noalloc)
//
// For callers that cannot call cudaMalloc once their scene is uploaded: a host
// application that hands the whole GPU memory budget to its own pool, or that
// forbids device allocation inside its frame loop.  The trace kernel's
// scratch — the persistent grid's ray counter, the work counters and the
// bounded-loop error word — and, for host buffers, the staging copies of the
// rays and hits live in one file-scope __device__ array instead of memory
// from cudaMalloc.  Its size is fixed: 256 bytes of launch state plus room for
// kNoAllocMaxRays rays and hits (1 MiB + 256 B in all).  A device holds it
// from the first scene upload on that device (which looks its address up)
// until the process exits.
// ---------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoAllocMaxRays = 16384; // host-buffer calls: rays per call
constexpr size_t kNoAllocStateBytes = 256;  // one StreamSlot, padded
constexpr size_t kNoAllocBytes = kNoAllocStateBytes + kNoAllocMaxRays * (32 + sizeof(lrt_hit));
static_assert(sizeof(lrt::StreamSlot) <= kNoAllocStateBytes, "launch state fits its 256 bytes");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

} // namespace

// The array's device address for the current device.  The symbol's name is
// only a host-side stand-in for the array and must never reach a kernel.
cudaError_t lrt::noalloc_scratch_address(void** p) { return cudaGetSymbolAddress(p, g_noalloc_scratch); }

extern "C" lrt_status lrt_trace_nearest_noalloc(lrt_scene* s, const float* rays, lrt_hit* hits, uint64_t n,
                                                void* stream_p, uint32_t flags)
{
  using namespace lrt;
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->committed || !s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "trace before CommitScene/upload");
  if (n == 0) return LRT_OK;
  if (!rays || !hits) return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_trace_nearest_noalloc: NULL rays or hits");
  if (flags & LRT_TRACE_COUNT_WORK)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_trace_nearest_noalloc: LRT_TRACE_COUNT_WORK is not supported");
  const bool onDevice = (flags & LRT_TRACE_DEVICE_POINTERS) != 0;
  if (!onDevice && n > kNoAllocMaxRays)
    return fail(s, LRT_ERR_INVALID_ARGUMENT,
                "lrt_trace_nearest_noalloc: %llu rays exceed the static scratch capacity of %llu rays per call",
                (unsigned long long)n, (unsigned long long)kNoAllocMaxRays);
  if (onDevice && ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "device rays/hits must be 16-byte aligned");
  lrt_status st = check_preset(s);
  if (st != LRT_OK) return st;
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaGetDevice");
  if (dev != s->device)
    return fail(s, LRT_ERR_INVALID_ARGUMENT,
                "lrt_trace_nearest_noalloc: make the scene's device (%d) current, not %d", s->device, dev);
  if (!s->dev->noallocBase)
    return fail(s, LRT_ERR_CUDA, "lrt_trace_nearest_noalloc: the static scratch array was not found at upload: %s",
                cudaGetErrorString(s->dev->noallocErr));
  unsigned char* base = s->dev->noallocBase;
  StreamSlot* slot = reinterpret_cast<StreamSlot*>(base);
  float4* srays = reinterpret_cast<float4*>(base + kNoAllocStateBytes);
  lrt_hit* shits = reinterpret_cast<lrt_hit*>(base + kNoAllocStateBytes + kNoAllocMaxRays * 32);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  DeviceScene* d = s->dev;
  DevScene S = d->S;
  S.flags = launch_flags(s);
  S.voxelStepCap = s->voxelStepCap ? s->voxelStepCap : kMaxVoxelSteps;
  // the array keeps the previous call's contents: the ray counter and the
  // error word must start at zero
  e = cudaMemsetAsync(slot, 0, sizeof(StreamSlot), stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaMemsetAsync(static scratch)");
  const float4* krays = onDevice ? reinterpret_cast<const float4*>(rays) : srays;
  lrt_hit* khits = onDevice ? hits : shits;
  if (!onDevice) {
    e = cudaMemcpyAsync(srays, rays, n * 32, cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "rays host->static scratch");
  }
  const uint64_t warps = (n + 31) / 32;
  const int grid = int(std::min<uint64_t>(uint64_t(d->grid), (warps * 32 + kTraceThreads - 1) / kTraceThreads));
  if (flags & LRT_TRACE_FAST_MATH)
    e = lrt_fast::launch_trace(S, krays, khits, n, &slot->work, slot->counters, &slot->err, d->stackCap, grid,
                               stream, false);
  else
    e = lrt_exact::launch_trace(S, krays, khits, n, &slot->work, slot->counters, &slot->err, d->stackCap, grid,
                                stream, false);
  if (e != cudaSuccess) return cuda_fail(s, e, "trace launch");
  if (!onDevice) {
    e = cudaMemcpyAsync(hits, shits, n * sizeof(lrt_hit), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "hits static scratch->host");
  }
  uint32_t err = 0;
  e = cudaMemcpyAsync(&err, &slot->err, sizeof(err), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "trace");
  if (err)
    return fail(s, LRT_ERR_DEVICE_LIMIT,
                "trace hit a bounded-loop limit (error bits 0x%x: 1 = stack, 2 = voxel march, 4 = transparency layers)", err);
  return LRT_OK;
}

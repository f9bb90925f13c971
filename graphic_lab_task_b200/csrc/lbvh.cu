// lbvh.cu — the device tree builder behind the BUILD_LOW build quality
// (CrossRT/CrossRT.h:14-17).  A linear BVH in the manner of Karras 2012
// ("Maximizing parallelism in the construction of BVHs, octrees, and k-d
// trees"): 30-bit Morton codes of the box centres, a radix sort, one thread per
// inner node of the binary radix tree over the sorted codes, and the inner
// boxes fitted bottom-up with one thread per leaf (the second child to arrive
// at a node fits it).  The host turns the tree into the reference's node
// layouts (fat BLAS pairs, the escape-index TLAS) with the same emitters as
// its SAH builder, so the arrays the traversal reads have the same format
// either way; only the tree shape differs.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>

#include <cub/device/device_radix_sort.cuh>

#include "lbvh.h"

namespace lrt {
namespace {

constexpr uint32_t kLeafFlag = 0x80000000u;
constexpr int kBlock = 256;
constexpr int kMaxClimb = 256; // tree depth bound of the bottom-up pass (a 62-bit key gives at most 63)

// Order-preserving map of floats to unsigned ints, for atomicMin/atomicMax.
__device__ __forceinline__ uint32_t float_key(float f)
{
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k)
{
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__global__ void k_init_bounds(uint32_t* bounds)
{
  if (threadIdx.x < 3) bounds[threadIdx.x] = 0xFFFFFFFFu;
  else if (threadIdx.x < 6) bounds[threadIdx.x] = 0u;
}

// Bounds of the box centres (NaN centres are left out).
__global__ void k_centre_bounds(const float* __restrict__ boxes, uint32_t n, uint32_t* bounds)
{
  const float inf = __int_as_float(0x7f800000);
  float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* b = boxes + 6 * uint64_t(i);
    for (int k = 0; k < 3; k++) {
      const float c = 0.5f * (b[k] + b[3 + k]);
      lo[k] = fminf(lo[k], c);
      hi[k] = fmaxf(hi[k], c);
    }
  }
  for (int k = 0; k < 3; k++)
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) {
      if (lo[k] <= hi[k]) {
        atomicMin(bounds + k, float_key(lo[k]));
        atomicMax(bounds + 3 + k, float_key(hi[k]));
      }
    }
}

// 10 bits per axis spread to every third bit.
__device__ __forceinline__ uint32_t spread10(uint32_t v)
{
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_morton(const float* __restrict__ boxes, uint32_t n, const uint32_t* __restrict__ bounds,
                         uint32_t* __restrict__ codes, uint32_t* __restrict__ ids)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* b = boxes + 6 * uint64_t(i);
  uint32_t q[3];
  for (int k = 0; k < 3; k++) {
    const float lo = key_float(bounds[k]), hi = key_float(bounds[3 + k]);
    const float ext = hi - lo;
    const float c = 0.5f * (b[k] + b[3 + k]);
    const float u = ext > 0.0f ? (c - lo) / ext : 0.0f;
    q[k] = uint32_t(fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f)); // NaN -> 0
  }
  codes[i] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
  ids[i] = i;
}

// Length of the common prefix of sorted keys i and j; equal codes are told
// apart by their positions (Karras 2012, section 4), -1 outside [0, n).
__device__ __forceinline__ int delta(const uint32_t* codes, uint32_t n, int i, int j)
{
  if (j < 0 || j >= int(n)) return -1;
  const uint32_t a = codes[i], b = codes[j];
  if (a != b) return __clz(a ^ b);
  return 32 + __clz(uint32_t(i) ^ uint32_t(j));
}

// One thread per inner node i of the radix tree over n sorted keys
// (Karras 2012, figure 4): its key range [first, last] and the split γ.
__global__ void k_radix_tree(const uint32_t* __restrict__ codes, uint32_t n, LbvhInner* __restrict__ inner,
                             uint32_t* __restrict__ parentLeaf, uint32_t* __restrict__ parentInner)
{
  const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= int(n) - 1) return;
  const int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = delta(codes, n, i, i - d);
  int lmax = 2;
  while (delta(codes, n, i, i + lmax * d) > dmin) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2)
    if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = delta(codes, n, i, j);
  int s = 0;
  for (int div = 2;; div *= 2) {
    const int t = (l + div - 1) / div;
    if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  const int g = i + s * d + (d < 0 ? -1 : 0);
  const int first = min(i, j), last = max(i, j);
  LbvhInner& node = inner[i];
  node.first = uint32_t(first);
  node.last = uint32_t(last);
  if (first == g) {
    node.kid[0] = uint32_t(g) | kLeafFlag;
    parentLeaf[g] = uint32_t(i);
  } else {
    node.kid[0] = uint32_t(g);
    parentInner[g] = uint32_t(i);
  }
  if (last == g + 1) {
    node.kid[1] = uint32_t(g + 1) | kLeafFlag;
    parentLeaf[g + 1] = uint32_t(i);
  } else {
    node.kid[1] = uint32_t(g + 1);
    parentInner[g + 1] = uint32_t(i);
  }
}

__device__ __forceinline__ void load_box(const float* __restrict__ boxes, const uint32_t* __restrict__ ids,
                                         const LbvhInner* inner, uint32_t kid, float* lo, float* hi)
{
  if (kid & kLeafFlag) {
    const float* b = boxes + 6 * uint64_t(ids[kid & ~kLeafFlag]);
    for (int k = 0; k < 3; k++) {
      lo[k] = b[k];
      hi[k] = b[3 + k];
    }
  } else {
    // written by another thread of this launch: read past L1
    const float* b = &inner[kid].lo[0];
    for (int k = 0; k < 3; k++) {
      lo[k] = __ldcg(b + k);
      hi[k] = __ldcg(b + 3 + k);
    }
  }
}

// One thread per leaf climbs towards the root; at each inner node the first
// arrival stops and the second fits the node's box to its two children.
__global__ void k_fit_boxes(const float* __restrict__ boxes, const uint32_t* __restrict__ ids, uint32_t n,
                            LbvhInner* inner, const uint32_t* __restrict__ parentLeaf,
                            const uint32_t* __restrict__ parentInner, uint32_t* arrivals, uint32_t* err)
{
  const uint32_t leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  uint32_t p = parentLeaf[leaf];
  for (int step = 0; step < kMaxClimb; step++) {
    __threadfence();
    if (atomicAdd(arrivals + p, 1u) == 0) return;
    __threadfence();
    float lo0[3], hi0[3], lo1[3], hi1[3];
    load_box(boxes, ids, inner, inner[p].kid[0], lo0, hi0);
    load_box(boxes, ids, inner, inner[p].kid[1], lo1, hi1);
    for (int k = 0; k < 3; k++) {
      __stcg(&inner[p].lo[k], fminf(lo0[k], lo1[k]));
      __stcg(&inner[p].hi[k], fmaxf(hi0[k], hi1[k]));
    }
    if (p == 0) return;
    p = parentInner[p];
  }
  atomicOr(err, 1u);
}

// Per-device scratch of the builds, reused while large enough.
struct ArenaCache {
  void* ptr = nullptr;
  size_t size = 0;
};
std::map<int, ArenaCache> g_arena;
std::mutex g_arenaMutex;

// Carves 256-byte-aligned pieces out of one device allocation.
struct Arena {
  size_t used = 0;
  char* base = nullptr;
  template <class T>
  T* take(size_t count)
  {
    T* p = reinterpret_cast<T*>(base + used);
    used += (count * sizeof(T) + 255) & ~size_t(255);
    return p;
  }
};

} // namespace

const char* lbvh_build(const float* boxes6, uint32_t n, std::vector<uint32_t>& order, std::vector<LbvhInner>& inner)
{
  order.clear();
  inner.clear();
  if (n == 0) return "no boxes";
  const char* what = nullptr;
  cudaError_t e = cudaSuccess;
  size_t tempBytes = 0;
  const uint32_t m = n > 1 ? n - 1 : 1;
  const unsigned blocks = (n + kBlock - 1) / kBlock;
#define LBVH_TRY(call, msg)                                                                                          \
  if (e == cudaSuccess) {                                                                                            \
    e = (call);                                                                                                      \
    if (e != cudaSuccess) what = msg;                                                                                \
  }
  {
    cub::DoubleBuffer<uint32_t> k0(nullptr, nullptr), v0(nullptr, nullptr);
    LBVH_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, k0, v0, int(n), 0, 30), "sort size");
  }
  // one allocation: a sizing pass over the same layout, then the real one
  Arena A;
  auto carve = [&](Arena& a) {
    struct P {
      float* boxes;
      uint32_t *bounds, *codes, *codesAlt, *ids, *idsAlt, *parentLeaf, *parentInner, *arrivals, *err;
      LbvhInner* inner;
      void* temp;
    } p;
    p.boxes = a.take<float>(6 * size_t(n));
    p.bounds = a.take<uint32_t>(8);
    p.codes = a.take<uint32_t>(n);
    p.codesAlt = a.take<uint32_t>(n);
    p.ids = a.take<uint32_t>(n);
    p.idsAlt = a.take<uint32_t>(n);
    p.inner = a.take<LbvhInner>(m);
    p.parentLeaf = a.take<uint32_t>(n);
    p.parentInner = a.take<uint32_t>(m);
    p.arrivals = a.take<uint32_t>(m);
    p.err = a.take<uint32_t>(1);
    p.temp = a.take<char>(tempBytes);
    return p;
  };
  carve(A);
  // the scratch of the largest build so far stays allocated per device, so
  // that repeated builds (dynamic meshes, TLAS rebuilds) do not pay for
  // cudaMalloc/cudaFree every time
  std::lock_guard<std::mutex> lock(g_arenaMutex);
  int dev = 0;
  LBVH_TRY(cudaGetDevice(&dev), "cudaGetDevice");
  void* arena = nullptr;
  if (e == cudaSuccess) {
    ArenaCache& ac = g_arena[dev];
    if (ac.size < A.used) {
      cudaFree(ac.ptr);
      ac.ptr = nullptr;
      ac.size = 0;
      LBVH_TRY(cudaMalloc(&ac.ptr, A.used), "device memory for the tree build");
      if (e == cudaSuccess) ac.size = A.used;
    }
    arena = ac.ptr;
  }
  A.base = static_cast<char*>(arena);
  A.used = 0;
  const auto P = carve(A);
  float* dBoxes = P.boxes;
  uint32_t *dBounds = P.bounds, *dCodes = P.codes, *dCodesAlt = P.codesAlt, *dIds = P.ids, *dIdsAlt = P.idsAlt;
  uint32_t *dParentLeaf = P.parentLeaf, *dParentInner = P.parentInner, *dArrivals = P.arrivals, *dErr = P.err;
  LbvhInner* dInner = P.inner;
  void* dTemp = P.temp;
  cudaStream_t st = nullptr;
  LBVH_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  LBVH_TRY(cudaMemcpyAsync(dBoxes, boxes6, 6 * sizeof(float) * size_t(n), cudaMemcpyHostToDevice, st),
           "boxes host->device");
  LBVH_TRY(cudaMemsetAsync(dArrivals, 0, sizeof(uint32_t) * m, st), "memset");
  LBVH_TRY(cudaMemsetAsync(dErr, 0, sizeof(uint32_t), st), "memset");
  if (e == cudaSuccess) {
    k_init_bounds<<<1, 32, 0, st>>>(dBounds);
    k_centre_bounds<<<std::min(blocks, 1184u), kBlock, 0, st>>>(dBoxes, n, dBounds);
    k_morton<<<blocks, kBlock, 0, st>>>(dBoxes, n, dBounds, dCodes, dIds);
    e = cudaGetLastError();
    if (e != cudaSuccess) what = "Morton code kernels";
  }
  cub::DoubleBuffer<uint32_t> keys(dCodes, dCodesAlt), vals(dIds, dIdsAlt);
  LBVH_TRY(cub::DeviceRadixSort::SortPairs(dTemp, tempBytes, keys, vals, int(n), 0, 30, st), "radix sort");
  if (e == cudaSuccess && n > 1) {
    k_radix_tree<<<(m + kBlock - 1) / kBlock, kBlock, 0, st>>>(keys.Current(), n, dInner, dParentLeaf,
                                                              dParentInner);
    k_fit_boxes<<<blocks, kBlock, 0, st>>>(dBoxes, vals.Current(), n, dInner, dParentLeaf, dParentInner, dArrivals,
                                           dErr);
    e = cudaGetLastError();
    if (e != cudaSuccess) what = "tree kernels";
  }
  uint32_t herr = 0;
  if (e == cudaSuccess) {
    order.resize(n);
    if (n > 1) inner.resize(n - 1);
  }
  LBVH_TRY(cudaMemcpyAsync(order.data(), vals.Current(), sizeof(uint32_t) * size_t(n), cudaMemcpyDeviceToHost, st),
           "order device->host");
  if (n > 1)
    LBVH_TRY(cudaMemcpyAsync(inner.data(), dInner, sizeof(LbvhInner) * size_t(n - 1), cudaMemcpyDeviceToHost, st),
             "tree device->host");
  LBVH_TRY(cudaMemcpyAsync(&herr, dErr, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "status device->host");
  LBVH_TRY(cudaStreamSynchronize(st), "tree build");
#undef LBVH_TRY
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    order.clear();
    inner.clear();
    static thread_local char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what ? what : "device tree build", cudaGetErrorString(e));
    return msg;
  }
  if (herr) {
    order.clear();
    inner.clear();
    return "device tree build: bottom-up pass exceeded its depth bound";
  }
  return nullptr;
}

} // namespace lrt

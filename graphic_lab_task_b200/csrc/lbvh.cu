// lbvh.cu — the device tree builder behind the BUILD_LOW build quality
// (CrossRT/CrossRT.h:14-17).  A linear BVH in the manner of Karras 2012
// ("Maximizing parallelism in the construction of BVHs, octrees, and k-d
// trees"): 30-bit Morton codes of the box centres, a radix sort, one thread per
// inner node of the binary radix tree over the sorted codes, and the inner
// boxes fitted bottom-up with one thread per leaf (the second child to arrive
// at a node fits it).  A triangle BLAS is then emitted on the device in the
// reference's fat-pair layout (lbvh_build_blas); the host turns the other
// trees (custom-box BLAS, the escape-index TLAS) into their layouts with the
// same emitters as its SAH builder.  The arrays the traversal reads have the
// same format either way; only the tree shape differs.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "lbvh.h"

namespace lrt {
namespace {

constexpr uint32_t kLeafFlag = 0x80000000u;
constexpr uint32_t kLeafWordBit = 0x80000000u;    // LEAF_BIT of a packed leaf word
constexpr uint32_t kEscapeRootWord = 0xFFFFFFFEu; // the root pair's escape word (emit_pairs)
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

// ---------------------------------------------------------------------------
// Emission of a triangle BLAS on the device, in the order of the host
// emitter (emit_pairs over the collapsed tree): node pairs in depth-first
// pre-order with the left subtree first; leaf ids in the order the pairs are
// created, a pair's left leaf before its right one; each leaf's triangles at
// the next free place of the triangle order; escape words of AlignNodes2
// (left node -> 2k+1, right node -> the parent's).  An inner node of the
// radix tree is emitted as a pair iff it holds more than maxLeaf boxes (all
// its ancestors do too); a child is a leaf if it is a box or an inner node
// of at most maxLeaf boxes.

__device__ __forceinline__ uint32_t kid_count(const LbvhInner* inner, uint32_t kid)
{
  return (kid & kLeafFlag) ? 1u : inner[kid].last - inner[kid].first + 1u;
}

// Pairs in each subtree (E), bottom-up: the second child to arrive at a node
// computes it, as k_fit_boxes fits the box.
__global__ void k_count_pairs(const LbvhInner* __restrict__ inner, uint32_t n, uint32_t maxLeaf,
                              const uint32_t* __restrict__ parentLeaf, const uint32_t* __restrict__ parentInner,
                              uint32_t* arrivals, uint32_t* pairsIn, uint32_t* err)
{
  const uint32_t leaf = blockIdx.x * blockDim.x + threadIdx.x;
  if (leaf >= n) return;
  uint32_t p = parentLeaf[leaf];
  for (int step = 0; step < kMaxClimb; step++) {
    __threadfence();
    if (atomicAdd(arrivals + p, 1u) == 0) return;
    __threadfence();
    const LbvhInner& in = inner[p];
    uint32_t e = 0;
    if (in.last - in.first + 1u > maxLeaf) {
      e = 1;
      for (int c = 0; c < 2; c++)
        if (!(in.kid[c] & kLeafFlag)) e += __ldcg(pairsIn + in.kid[c]);
    }
    __stcg(pairsIn + p, e);
    if (p == 0) return;
    p = parentInner[p];
  }
  atomicOr(err, 1u);
}

// Pre-order index and parent escape word of every emitted node (a climb to
// the root summing the offsets of the left subtrees passed), and the number
// of its leaf children at its index.
__global__ void k_preorder(const LbvhInner* __restrict__ inner, uint32_t m, uint32_t maxLeaf,
                           const uint32_t* __restrict__ parentInner, const uint32_t* __restrict__ pairsIn,
                           uint32_t* __restrict__ pre, uint32_t* __restrict__ esc, uint32_t* __restrict__ leafKids,
                           uint32_t* err)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const LbvhInner& in = inner[i];
  if (in.last - in.first + 1u <= maxLeaf) return;
  uint32_t acc = 0, escAcc = 0;
  bool left = false;
  uint32_t c = i;
  int step = 0;
  for (; c != 0 && step < kMaxClimb; step++) {
    const uint32_t p = parentInner[c];
    const LbvhInner& P = inner[p];
    if (P.kid[0] == c) {
      acc += 1;
      if (!left) {
        left = true;
        escAcc = acc; // pre(i) - pre(p)
      }
    } else {
      const uint32_t l = P.kid[0];
      acc += 1 + ((l & kLeafFlag) ? 0u : pairsIn[l]);
    }
    c = p;
  }
  if (c != 0 || acc >= m) {
    atomicOr(err, 2u);
    return;
  }
  pre[i] = acc;
  esc[i] = left ? 2u * (acc - escAcc) + 1u : kEscapeRootWord;
  uint32_t lk = 0;
  for (int k = 0; k < 2; k++)
    if (kid_count(inner, in.kid[k]) <= maxLeaf) lk++;
  leafKids[acc] = lk;
}

// Each emitted node's leaf children: their ids (from the scanned leaf-child
// counts), triangle counts and first sorted positions, by leaf id.
__global__ void k_leaves(const LbvhInner* __restrict__ inner, uint32_t m, uint32_t n, uint32_t maxLeaf,
                         const uint32_t* __restrict__ pre, const uint32_t* __restrict__ leafBase,
                         uint32_t* __restrict__ leafCount, uint32_t* __restrict__ leafFirst)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const LbvhInner& in = inner[i];
  if (in.last - in.first + 1u <= maxLeaf || pre[i] >= m) return;
  uint32_t id = leafBase[pre[i]];
  for (int k = 0; k < 2; k++) {
    const uint32_t kid = in.kid[k];
    const uint32_t cnt = kid_count(inner, kid);
    if (cnt > maxLeaf) continue;
    if (id >= n) return; // an inconsistent tree; k_totals' bound check reports it
    leafCount[id] = cnt;
    leafFirst[id] = (kid & kLeafFlag) ? (kid & ~kLeafFlag) : inner[kid].first;
    id++;
  }
}

__device__ __forceinline__ uint32_t leaf_word(uint32_t start, uint32_t size)
{
  return kLeafWordBit | ((size << 28) & 0x70000000u) | (start & 0x0FFFFFFFu); // raytrace_common.h:51-54
}

// The pairs: the children's boxes, child words (pre-order index of an
// emitted child, Pack(leafId, 1) of a leaf), escape words.
__global__ void k_emit_pairs(const float* __restrict__ boxes, const uint32_t* __restrict__ ids,
                             const LbvhInner* __restrict__ inner, uint32_t m, uint32_t maxLeaf,
                             const uint32_t* __restrict__ pre, const uint32_t* __restrict__ esc,
                             const uint32_t* __restrict__ leafBase, LbvhPairOut* __restrict__ pairs)
{
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const LbvhInner& in = inner[i];
  if (in.last - in.first + 1u <= maxLeaf) return;
  const uint32_t k = pre[i];
  if (k >= m) return;
  uint32_t id = leafBase[k];
  LbvhPairOut out;
  for (int c = 0; c < 2; c++) {
    const uint32_t kid = in.kid[c];
    float lo[3], hi[3];
    if (kid & kLeafFlag) {
      const float* b = boxes + 6 * uint64_t(ids[kid & ~kLeafFlag]);
      for (int a = 0; a < 3; a++) {
        lo[a] = b[a];
        hi[a] = b[3 + a];
      }
    } else {
      for (int a = 0; a < 3; a++) {
        lo[a] = inner[kid].lo[a];
        hi[a] = inner[kid].hi[a];
      }
    }
    uint32_t word;
    if (kid_count(inner, kid) > maxLeaf) {
      word = pre[kid];
    } else {
      word = leaf_word(id, 1);
      id++;
    }
    float* node = out.node[c];
    for (int a = 0; a < 3; a++) {
      node[a] = lo[a];
      node[4 + a] = hi[a];
    }
    node[3] = __uint_as_float(word);
    node[7] = __uint_as_float(c == 0 ? 2u * k + 1u : esc[i]);
  }
  pairs[k] = out;
}

// The leaf table (Pack(start, count) per leaf id) and the triangle order.
// One thread per possible leaf id l < n (ids past the last leaf have count 0).
__global__ void k_leaf_table(const uint32_t* __restrict__ ids, uint32_t n, const uint32_t* __restrict__ leafCount,
                             const uint32_t* __restrict__ leafFirst, const uint32_t* __restrict__ leafStart,
                             uint32_t* __restrict__ startCount, uint32_t* __restrict__ order)
{
  const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= n) return;
  const uint32_t cnt = leafCount[l], start = leafStart[l], first = leafFirst[l];
  startCount[l] = leaf_word(start, cnt);
  if (cnt == 0 || uint64_t(start) + cnt > n || uint64_t(first) + cnt > n) return;
  for (uint32_t j = 0; j < cnt; j++) order[start + j] = ids[first + j];
}

// {pairs, leaves}: the root's pair count, and the leaf ids handed out.
__global__ void k_totals(const uint32_t* __restrict__ pairsIn, const uint32_t* __restrict__ leafBase,
                         const uint32_t* __restrict__ leafKids, uint32_t* totals)
{
  const uint32_t P = pairsIn[0];
  totals[0] = P;
  totals[1] = P ? leafBase[P - 1] + leafKids[P - 1] : 0u;
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

namespace {

// The build on the current device; with `emit` (maxLeaf > 0) the triangle
// BLAS emission too.  Outputs: order and, without emission, the inner nodes;
// with it, the pairs and leaf table (order then being the leaves' box order).
const char* run(const float* boxes6, uint32_t n, uint32_t maxLeaf, bool emit, std::vector<uint32_t>& order,
                std::vector<LbvhInner>* innerOut, const std::function<LbvhPairOut*(size_t)>* pairsAt,
                std::vector<uint32_t>* startCountOut)
{
  order.clear();
  if (innerOut) innerOut->clear();
  if (startCountOut) startCountOut->clear();
  if (n == 0) return "no boxes";
  if (emit && n <= maxLeaf) return "device emission of a single-leaf tree";
  const char* what = nullptr;
  cudaError_t e = cudaSuccess;
  size_t tempBytes = 0, scanBytes = 0;
  const uint32_t m = n > 1 ? n - 1 : 1;
  const unsigned blocks = (n + kBlock - 1) / kBlock;
  const unsigned innerBlocks = (m + kBlock - 1) / kBlock;
#define LBVH_TRY(call, msg)                                                                                          \
  if (e == cudaSuccess) {                                                                                            \
    e = (call);                                                                                                      \
    if (e != cudaSuccess) what = msg;                                                                                \
  }
  {
    cub::DoubleBuffer<uint32_t> k0(nullptr, nullptr), v0(nullptr, nullptr);
    LBVH_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, k0, v0, int(n), 0, 30), "sort size");
    if (emit) {
      uint32_t* none = nullptr;
      LBVH_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, none, none, int(n)), "scan size");
    }
  }
  // one allocation: a sizing pass over the same layout, then the real one
  Arena A;
  auto carve = [&](Arena& a) {
    struct P {
      float* boxes;
      uint32_t *bounds, *codes, *codesAlt, *ids, *idsAlt, *parentLeaf, *parentInner, *arrivals, *err;
      LbvhInner* inner;
      void* temp;
      // emission
      uint32_t *pairsIn, *pre, *esc, *leafKids, *leafBase, *leafCount, *leafFirst, *leafStart, *startCount, *order,
          *totals;
      LbvhPairOut* pairs;
      void* scanTemp;
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
    const size_t em = emit ? m : 0, en = emit ? n : 0;
    p.pairsIn = a.take<uint32_t>(em);
    p.pre = a.take<uint32_t>(em);
    p.esc = a.take<uint32_t>(em);
    p.leafKids = a.take<uint32_t>(em);
    p.leafBase = a.take<uint32_t>(em);
    p.leafCount = a.take<uint32_t>(en);
    p.leafFirst = a.take<uint32_t>(en);
    p.leafStart = a.take<uint32_t>(en);
    p.startCount = a.take<uint32_t>(en);
    p.order = a.take<uint32_t>(en);
    p.totals = a.take<uint32_t>(emit ? 2 : 0);
    p.pairs = a.take<LbvhPairOut>(em);
    p.scanTemp = a.take<char>(emit ? scanBytes : 0);
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
  cudaStream_t st = nullptr;
  LBVH_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  LBVH_TRY(cudaMemcpyAsync(P.boxes, boxes6, 6 * sizeof(float) * size_t(n), cudaMemcpyHostToDevice, st),
           "boxes host->device");
  LBVH_TRY(cudaMemsetAsync(P.arrivals, 0, sizeof(uint32_t) * m, st), "memset");
  LBVH_TRY(cudaMemsetAsync(P.err, 0, sizeof(uint32_t), st), "memset");
  if (e == cudaSuccess) {
    k_init_bounds<<<1, 32, 0, st>>>(P.bounds);
    k_centre_bounds<<<std::min(blocks, 1184u), kBlock, 0, st>>>(P.boxes, n, P.bounds);
    k_morton<<<blocks, kBlock, 0, st>>>(P.boxes, n, P.bounds, P.codes, P.ids);
    e = cudaGetLastError();
    if (e != cudaSuccess) what = "Morton code kernels";
  }
  cub::DoubleBuffer<uint32_t> keys(P.codes, P.codesAlt), vals(P.ids, P.idsAlt);
  LBVH_TRY(cub::DeviceRadixSort::SortPairs(P.temp, tempBytes, keys, vals, int(n), 0, 30, st), "radix sort");
  if (e == cudaSuccess && n > 1) {
    k_radix_tree<<<innerBlocks, kBlock, 0, st>>>(keys.Current(), n, P.inner, P.parentLeaf, P.parentInner);
    k_fit_boxes<<<blocks, kBlock, 0, st>>>(P.boxes, vals.Current(), n, P.inner, P.parentLeaf, P.parentInner,
                                           P.arrivals, P.err);
    e = cudaGetLastError();
    if (e != cudaSuccess) what = "tree kernels";
  }
  uint32_t herr = 0, totals[2] = {0, 0};
  if (emit) {
    // n > maxLeaf >= 1: the root is an emitted inner node
    LBVH_TRY(cudaMemsetAsync(P.arrivals, 0, sizeof(uint32_t) * m, st), "memset");
    LBVH_TRY(cudaMemsetAsync(P.leafKids, 0, sizeof(uint32_t) * m, st), "memset");
    LBVH_TRY(cudaMemsetAsync(P.pre, 0xFF, sizeof(uint32_t) * m, st), "memset");
    if (e == cudaSuccess) {
      k_count_pairs<<<blocks, kBlock, 0, st>>>(P.inner, n, maxLeaf, P.parentLeaf, P.parentInner, P.arrivals,
                                                P.pairsIn, P.err);
      k_preorder<<<innerBlocks, kBlock, 0, st>>>(P.inner, m, maxLeaf, P.parentInner, P.pairsIn, P.pre, P.esc,
                                                 P.leafKids, P.err);
      e = cudaGetLastError();
      if (e != cudaSuccess) what = "pair numbering kernels";
    }
    LBVH_TRY(cub::DeviceScan::ExclusiveSum(P.scanTemp, scanBytes, P.leafKids, P.leafBase, int(m), st), "leaf scan");
    LBVH_TRY(cudaMemsetAsync(P.leafCount, 0, sizeof(uint32_t) * n, st), "memset");
    if (e == cudaSuccess) {
      k_leaves<<<innerBlocks, kBlock, 0, st>>>(P.inner, m, n, maxLeaf, P.pre, P.leafBase, P.leafCount, P.leafFirst);
      e = cudaGetLastError();
      if (e != cudaSuccess) what = "leaf kernel";
    }
    LBVH_TRY(cub::DeviceScan::ExclusiveSum(P.scanTemp, scanBytes, P.leafCount, P.leafStart, int(n), st),
             "triangle scan");
    if (e == cudaSuccess) {
      k_totals<<<1, 1, 0, st>>>(P.pairsIn, P.leafBase, P.leafKids, P.totals);
      k_emit_pairs<<<innerBlocks, kBlock, 0, st>>>(P.boxes, vals.Current(), P.inner, m, maxLeaf, P.pre, P.esc,
                                                   P.leafBase, P.pairs);
      k_leaf_table<<<blocks, kBlock, 0, st>>>(vals.Current(), n, P.leafCount, P.leafFirst, P.leafStart,
                                              P.startCount, P.order);
      e = cudaGetLastError();
      if (e != cudaSuccess) what = "emission kernels";
    }
    LBVH_TRY(cudaMemcpyAsync(totals, P.totals, sizeof(totals), cudaMemcpyDeviceToHost, st), "totals device->host");
    LBVH_TRY(cudaMemcpyAsync(&herr, P.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "status device->host");
    LBVH_TRY(cudaStreamSynchronize(st), "tree emission");
    if (e == cudaSuccess && !herr && (totals[0] == 0 || totals[0] > m || totals[1] > n)) herr = 4;
    LbvhPairOut* pairsDst = nullptr;
    if (e == cudaSuccess && !herr) {
      pairsDst = (*pairsAt)(totals[0]);
      startCountOut->resize(totals[1]);
      order.resize(n);
    }
    if (!herr) {
      LBVH_TRY(cudaMemcpyAsync(pairsDst, P.pairs, sizeof(LbvhPairOut) * size_t(totals[0]), cudaMemcpyDeviceToHost,
                               st),
               "pairs device->host");
      LBVH_TRY(cudaMemcpyAsync(startCountOut->data(), P.startCount, sizeof(uint32_t) * size_t(totals[1]),
                               cudaMemcpyDeviceToHost, st),
               "leaf table device->host");
      LBVH_TRY(cudaMemcpyAsync(order.data(), P.order, sizeof(uint32_t) * size_t(n), cudaMemcpyDeviceToHost, st),
               "order device->host");
    }
  } else {
    if (e == cudaSuccess) {
      order.resize(n);
      if (n > 1) innerOut->resize(n - 1);
    }
    LBVH_TRY(cudaMemcpyAsync(order.data(), vals.Current(), sizeof(uint32_t) * size_t(n), cudaMemcpyDeviceToHost, st),
             "order device->host");
    if (n > 1)
      LBVH_TRY(cudaMemcpyAsync(innerOut->data(), P.inner, sizeof(LbvhInner) * size_t(n - 1), cudaMemcpyDeviceToHost,
                               st),
               "tree device->host");
    LBVH_TRY(cudaMemcpyAsync(&herr, P.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st), "status device->host");
  }
  LBVH_TRY(cudaStreamSynchronize(st), "tree build");
#undef LBVH_TRY
  if (st) cudaStreamDestroy(st);
  auto clear = [&]() { // (pairs the caller made room for are the caller's to drop)
    order.clear();
    if (innerOut) innerOut->clear();
    if (startCountOut) startCountOut->clear();
  };
  if (e != cudaSuccess) {
    clear();
    static thread_local char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what ? what : "device tree build", cudaGetErrorString(e));
    return msg;
  }
  if (herr) {
    clear();
    return (herr & 1u) ? "device tree build: bottom-up pass exceeded its depth bound"
                       : "device tree emission: inconsistent tree";
  }
  return nullptr;
}

} // namespace

const char* lbvh_build(const float* boxes6, uint32_t n, std::vector<uint32_t>& order, std::vector<LbvhInner>& inner)
{
  return run(boxes6, n, 0, false, order, &inner, nullptr, nullptr);
}

const char* lbvh_build_blas(const float* boxes6, uint32_t n, uint32_t maxLeaf,
                            const std::function<LbvhPairOut*(size_t)>& pairsAt, std::vector<uint32_t>& startCount,
                            std::vector<uint32_t>& order)
{
  return run(boxes6, n, std::max(1u, maxLeaf), true, order, nullptr, &pairsAt, &startCount);
}

} // namespace lrt

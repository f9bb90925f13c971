// embree_shim.cpp — stand-in for the six Embree 3 builder entry points that
// the reference BVH builder calls (utils/raytracing/cbvh_embree2.cpp:287-331).
//
// TEST INFRASTRUCTURE ONLY: linked into oracle/_ref/liblrt_ref.so, the
// reference build used as a checker.  libembree3.so.3 is absent from the
// reference tree (a missing blob), so this file restates the public contract
// of rtcBuildBVH from the Embree 3 headers shipped with the reference
// (dependencies/embree3/embree3/rtcore_builder.h):
//   - primitives are RTCBuildPrimitive boxes, the tree is built top-down,
//   - every inner node is created with createNode(alloc, 2, user), its
//     children attached with setNodeChildren and their boxes with
//     setNodeBounds, every leaf with createLeaf(alloc, prims, count, user),
//   - nodes live in memory handed out by rtcThreadLocalAlloc, owned by the
//     RTCBVH and released with it.
// The split choice is a plain binned SAH (32 bins per axis over primitive
// centroids), so trees are not Embree's; parity never depends on that,
// because the CPU reference and the GPU kernels traverse the same arrays.
#include <algorithm>
#include <cfloat>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "embree3/rtcore.h"

struct RTCDeviceTy {
  int refs = 1;
};

struct RTCThreadLocalAllocatorTy {
  std::vector<void*> blocks;
  void* alloc(size_t bytes, size_t align)
  {
    if (align < 16) align = 16;
    void* p = nullptr;
    if (posix_memalign(&p, align, bytes ? bytes : align) != 0) return nullptr;
    blocks.push_back(p);
    return p;
  }
  ~RTCThreadLocalAllocatorTy()
  {
    for (void* p : blocks) free(p);
  }
};

struct RTCBVHTy {
  int refs = 1;
  RTCThreadLocalAllocatorTy arena;
};

namespace {

struct Box {
  float lo[3], hi[3];
  void reset()
  {
    for (int k = 0; k < 3; k++) { lo[k] = FLT_MAX; hi[k] = -FLT_MAX; }
  }
  void grow(const Box& b)
  {
    for (int k = 0; k < 3; k++) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
  }
  float area() const
  {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
    return 2.0f * (dx * dy + dy * dz + dz * dx);
  }
};

struct Builder {
  const RTCBuildArguments* args;
  std::vector<Box> boxes;
  std::vector<float> cent[3];
  std::vector<uint32_t> ids;

  Box bounds(size_t b, size_t e) const
  {
    Box r;
    r.reset();
    for (size_t i = b; i < e; i++) r.grow(boxes[ids[i]]);
    return r;
  }

  size_t split(size_t b, size_t e)
  {
    constexpr int NB = 32;
    float cmin[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, cmax[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (size_t i = b; i < e; i++)
      for (int k = 0; k < 3; k++) {
        cmin[k] = std::min(cmin[k], cent[k][ids[i]]);
        cmax[k] = std::max(cmax[k], cent[k][ids[i]]);
      }
    float best = FLT_MAX;
    int bestAxis = -1, bestBin = 0;
    for (int k = 0; k < 3; k++) {
      const float ext = cmax[k] - cmin[k];
      if (!(ext > 0.0f)) continue;
      Box bb[NB];
      int cnt[NB] = {0};
      for (int i = 0; i < NB; i++) bb[i].reset();
      for (size_t i = b; i < e; i++) {
        int bin = int((cent[k][ids[i]] - cmin[k]) / ext * NB);
        bin = std::min(std::max(bin, 0), NB - 1);
        cnt[bin]++;
        bb[bin].grow(boxes[ids[i]]);
      }
      float rightArea[NB];
      int rightCnt[NB];
      Box acc;
      acc.reset();
      int c = 0;
      for (int i = NB - 1; i > 0; i--) {
        acc.grow(bb[i]);
        c += cnt[i];
        rightArea[i] = acc.area();
        rightCnt[i] = c;
      }
      acc.reset();
      c = 0;
      for (int i = 0; i < NB - 1; i++) {
        acc.grow(bb[i]);
        c += cnt[i];
        if (c == 0 || rightCnt[i + 1] == 0) continue;
        const float cost = acc.area() * c + rightArea[i + 1] * rightCnt[i + 1];
        if (cost < best) { best = cost; bestAxis = k; bestBin = i; }
      }
    }
    if (bestAxis < 0) return b + (e - b) / 2; // all centroids coincide: split by count
    const float ext = cmax[bestAxis] - cmin[bestAxis];
    auto mid = std::partition(ids.begin() + b, ids.begin() + e, [&](uint32_t id) {
      int bin = int((cent[bestAxis][id] - cmin[bestAxis]) / ext * NB);
      bin = std::min(std::max(bin, 0), NB - 1);
      return bin <= bestBin;
    });
    size_t m = size_t(mid - ids.begin());
    if (m == b || m == e) m = b + (e - b) / 2;
    return m;
  }

  void* build(size_t b, size_t e, RTCThreadLocalAllocator alloc)
  {
    const size_t maxLeaf = std::max<unsigned>(1u, args->maxLeafSize);
    if (e - b <= maxLeaf) {
      std::vector<RTCBuildPrimitive> prims(e - b);
      for (size_t i = b; i < e; i++) prims[i - b] = args->primitives[ids[i]];
      return args->createLeaf(alloc, prims.data(), prims.size(), args->userPtr);
    }
    const size_t m = split(b, e);
    void* node = args->createNode(alloc, 2, args->userPtr);
    void* kids[2] = {build(b, m, alloc), build(m, e, alloc)};
    RTCBounds bb[2];
    const size_t rb[2][2] = {{b, m}, {m, e}};
    for (int j = 0; j < 2; j++) {
      const Box x = bounds(rb[j][0], rb[j][1]);
      bb[j].lower_x = x.lo[0]; bb[j].lower_y = x.lo[1]; bb[j].lower_z = x.lo[2]; bb[j].align0 = 0.0f;
      bb[j].upper_x = x.hi[0]; bb[j].upper_y = x.hi[1]; bb[j].upper_z = x.hi[2]; bb[j].align1 = 0.0f;
    }
    const RTCBounds* bp[2] = {&bb[0], &bb[1]};
    args->setNodeChildren(node, kids, 2, args->userPtr);
    args->setNodeBounds(node, bp, 2, args->userPtr);
    return node;
  }
};

} // namespace

extern "C" {

RTCDevice rtcNewDevice(const char*) { return new RTCDeviceTy(); }
void rtcRetainDevice(RTCDevice d) { d->refs++; }
void rtcReleaseDevice(RTCDevice d)
{
  if (d && --d->refs == 0) delete d;
}
RTCBVH rtcNewBVH(RTCDevice) { return new RTCBVHTy(); }
void rtcRetainBVH(RTCBVH b) { b->refs++; }
void rtcReleaseBVH(RTCBVH b)
{
  if (b && --b->refs == 0) delete b;
}
void* rtcThreadLocalAlloc(RTCThreadLocalAllocator a, size_t bytes, size_t align) { return a->alloc(bytes, align); }

void* rtcBuildBVH(const RTCBuildArguments* args)
{
  if (!args || !args->bvh || args->primitiveCount == 0) return nullptr;
  Builder B;
  B.args = args;
  const size_t n = args->primitiveCount;
  B.boxes.resize(n);
  for (int k = 0; k < 3; k++) B.cent[k].resize(n);
  B.ids.resize(n);
  for (size_t i = 0; i < n; i++) {
    const RTCBuildPrimitive& p = args->primitives[i];
    Box& x = B.boxes[i];
    x.lo[0] = p.lower_x; x.lo[1] = p.lower_y; x.lo[2] = p.lower_z;
    x.hi[0] = p.upper_x; x.hi[1] = p.upper_y; x.hi[2] = p.upper_z;
    for (int k = 0; k < 3; k++) B.cent[k][i] = 0.5f * (x.lo[k] + x.hi[k]);
    B.ids[i] = uint32_t(i);
  }
  return B.build(0, n, &args->bvh->arena);
}

} // extern "C"

// trace_impl.cuh — sm_100a nearest-hit traversal (BVHRT::RayQuery_NearestHit).
//
// Included by trace_exact.cu (-fmad=false: bit-identical to the reference CPU
// build with -ffp-contract=off) and trace_fast.cu (FMA contraction on).  Each
// includer defines LRT_NS to put its copy of the kernels in its own namespace.
//
// Structure follows the reference path function by function:
//   trace_one        RayQuery_NearestHit        MultiRenderer/BVH2Common.cpp:3322-3392
//   blas             BVH2TraverseF32            :3239-3320
//   leaf             IntersectAllPrimitivesInLeaf :47-124
//   triangles        IntersectAllTrianglesInLeaf  :1571-1635
//   octree_node      OctreeNodeIntersect + RayNodeIntersection :727-749, 141-218
//   octree_brick     OctreeBrickIntersect + load_distance_values :884-1112, 846-882
//   local_surface    LocalSurfaceIntersection (ST/BBOX) :345-391, 618-690
// The device reads B200-specific layouts built at upload (device_layout.h):
// pre-gathered triangles (vertex A + two edges, 48 B), bricks resolved to
// dense (brick_size+1)^3 fp32 corner grids, and a 32-B per-geometry table.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_layout.h"
#include "lrt_math.h"

namespace LRT_NS {
using namespace lrt;

struct Counters {
  uint32_t c[LRT_COUNTER_COUNT];
};

// What the adjoint needs about the final hit when it lies on an indexed SBS
// brick: the 8 corner values and their indices in the float value array,
// the voxel-local hit point, the object-space direction and the voxel size.
struct HitRecord {
  float t;          // hit.t when recorded (the record is valid iff it equals the final hit.t)
  float values[8];
  uint32_t idx[8];
  f3 p;
  f3 dir;
  float d;
  bool sbs;         // set by octree_brick for the indexed layouts
  bool early;       // the field was already <= EPS where the ray entered the
                    // voxel: the hit is that entry point, which does not move
                    // with the values (no dt/dtheta term)
};

// Traversal context.  COUNT adds the work counters, RECORD the hit record,
// SOLVERS the ANALYTIC / NEWTON / IT node solvers (ST and BBOX are always
// there); the plain trace kernel instantiates none.  nrec points at this thread's
// kNormalWords shared-memory words (thread-strided), where a sphere-traced
// hit leaves what its normal is computed from once the traversal has ended.
template <bool COUNT, bool RECORD = false, bool SOLVERS = false>
struct Ctx {
  static constexpr bool kCount = COUNT;
  static constexpr bool kRecord = RECORD;
  static constexpr bool kSolvers = SOLVERS;
  const DevScene& S;
  float* nrec;
  Counters cnt;
  uint32_t err;
  uint32_t triLocal; // a triangle hit's primId before the m_primIndices remap (its triSoup record)
  HitRecord rec;
  __device__ Ctx(const DevScene& s, float* normal_rec) : S(s), nrec(normal_rec), err(0)
  {
#pragma unroll
    for (int i = 0; i < LRT_COUNTER_COUNT; i++) cnt.c[i] = 0;
    if (RECORD) {
      rec.t = -1.0f;
      rec.sbs = false;
    }
  }
  __device__ __forceinline__ void inc(int k, uint32_t v = 1)
  {
    if (COUNT) cnt.c[k] += v;
  }
};

__device__ __forceinline__ f3 ld3(const float4 v) { return mk3(v.x, v.y, v.z); }

// This thread's deferred-normal words: after a stack of stack_cap entries.
__device__ __forceinline__ float* normal_words(uint32_t* smem, uint32_t stack_cap)
{
  return reinterpret_cast<float*>(smem + stack_cap * blockDim.x) + threadIdx.x;
}

// The normal of LocalSurfaceIntersection (BVH2Common.cpp:652-680) from the
// words a hit left: sign, sample point (start_q in the BBOX mode) and corner
// values; normalised in world space and octahedrally encoded.
template <class CTX>
__device__ __forceinline__ f2 deferred_normal(CTX& c, uint32_t instId)
{
  const DevScene& S = c.S;
  const uint32_t st = blockDim.x;
  const float* w = c.nrec;
  const float start_sign = w[0];
  const f3 q = mk3(w[st], w[2 * st], w[3 * st]);
  f3 norm;
  if (S.flags & kFlagBBoxMode) { // every hit is an early hit in this mode
    const f3 v = mk3(smax(q.x, 1 - q.x), smax(q.y, 1 - q.y), smax(q.z, 1 - q.z));
    const float qa[3] = {q.x, q.y, q.z};
    int dim = 0;
    if (v.y > v.x && v.y > v.z) dim = 1;
    else if (v.z > v.x && v.z > v.y) dim = 2;
    float nn[3] = {0, 0, 0};
    nn[dim] = qa[dim] < 0.5f ? -1.0f : 1.0f;
    norm = mk3(nn[0], nn[1], nn[2]);
  } else {
    float values[8];
#pragma unroll
    for (int i = 0; i < 8; i++) values[i] = w[(4 + i) * st];
    const float h = 0.001f;
    const float ddx = (trilinear(values, q + mk3(h, 0, 0)) - trilinear(values, q + mk3(-h, 0, 0))) / (2 * h);
    const float ddy = (trilinear(values, q + mk3(0, h, 0)) - trilinear(values, q + mk3(0, -h, 0))) / (2 * h);
    const float ddz = (trilinear(values, q + mk3(0, 0, h)) - trilinear(values, q + mk3(0, 0, -h))) / (2 * h);
    norm = start_sign * mk3(ddx, ddy, ddz);
  }
  norm = normalize(matmul4(S.instances[instId].transformInvTransposed, norm, 1.0f));
  return encode_normal(norm);
}

// The cubic c3 t^3 + c2 t^2 + c1 t + c0 whose root is the trilinear surface
// along the ray inside one voxel, in voxel units (BVH2Common.cpp:395-436).
__device__ __forceinline__ void sdf_cubic(const float* values, float d_inv, f3 o, f3 d3, float* c)
{
  const float s000 = values[0] * d_inv, s001 = values[1] * d_inv, s010 = values[2] * d_inv;
  const float s011 = values[3] * d_inv, s100 = values[4] * d_inv, s101 = values[5] * d_inv;
  const float s110 = values[6] * d_inv, s111 = values[7] * d_inv;
  const float tmp = s101 - s001;
  const float k0 = s000;
  const float k1 = s100 - s000;
  const float k2 = s010 - s000;
  const float k3 = s110 - s010 - k1;
  const float k4 = k0 - s001;
  const float k5 = k1 - tmp;
  const float k6 = k2 - (s011 - s001);
  const float k7 = k3 - (s111 - s011 - tmp);
  const float m0 = o.x * o.y;
  const float m1 = d3.x * d3.y;
  const float m2 = o.x * d3.y + o.y * d3.x;
  const float m3 = k5 * o.z - k1;
  const float m4 = k6 * o.z - k2;
  const float m5 = k7 * o.z - k3;
  c[0] = (k4 * o.z - k0) + o.x * m3 + o.y * m4 + m0 * m5;
  c[1] = d3.x * m3 + d3.y * m4 + m2 * m5 + d3.z * (k4 + k5 * o.x + k6 * o.y + k7 * m0);
  c[2] = m1 * m5 + d3.z * (k5 * d3.x + k6 * d3.y + k7 * m2);
  c[3] = k7 * m1 * d3.z;
}

// ANALYTIC (BVH2Common.cpp:441-505): the smallest non-negative real root.
// The reference's unqualified sqrt is the C library's double sqrt, so the
// expressions containing it are evaluated in double; acos, pow and cos are
// CUDA's, which may differ from the host library's in the last bit.
__device__ __forceinline__ float sdf_root_analytic(const float* c, float EPS)
{
  const float c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
  const float kPi = 3.14159265358979323846f; // LiteMath::M_PI, a float
  float x1 = 1000, x2 = 1000, x3 = 1000;
  if (fabsf(c3) > 1e-5f) {
    const float a = c2 / c3, b = c1 / c3, cc = c0 / c3;
    const float Q = (a * a - 3 * b) / 9;
    const float R = (2 * a * a * a - 9 * a * b + 27 * cc) / 54;
    const float Q3 = Q * Q * Q;
    if (R * R < Q3) {
      const float theta = float(acos(double(R) / sqrt(double(Q3))));
      const double sQ = -2.0 * sqrt(double(Q));
      x1 = float(sQ * double(cosf(theta / 3)) - double(a / 3));
      x2 = float(sQ * double(cosf((theta + 2 * kPi) / 3)) - double(a / 3));
      x3 = float(sQ * double(cosf((theta - 2 * kPi) / 3)) - double(a / 3));
    } else {
      const float A = float(double(-ssign(R)) * pow(double(fabsf(R)) + sqrt(double(R * R - Q3)),
                                                     double(1.0f / 3.0f)));
      const float B = fabsf(A) > EPS ? Q / A : 0;
      x1 = A + B - a / 3;
    }
  } else if (fabsf(c2) > 1e-7f) {
    const float a = c2, b = c1, cc = c0;
    const float D = b * b - 4 * a * cc;
    if (D > 0) {
      const float q = -0.5f * (b + ssign(b) * sqrtf(D));
      x1 = q / a;
      if (fabsf(q) > EPS) x2 = cc / q;
    }
  } else if (fabsf(c1) > EPS) {
    x1 = -c0 / c1;
  }
  x1 = x1 < 0 ? 1000 : x1;
  x2 = x2 < 0 ? 1000 : x2;
  x3 = x3 < 0 ? 1000 : x3;
  return smin(x1, smin(x2, x3));
}

// NEWTON (BVH2Common.cpp:507-587): a sign change of the cubic bracketed by
// 0, the roots of its derivative and qFar, then at most 10 Newton steps.
__device__ __forceinline__ bool sdf_root_newton(const float* c, float qFar, float EPS, float& t)
{
  const float c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
  const float a = 3 * c3, b = 2 * c2, cc = c1;
  const float t0 = 0;
  float t1 = qFar, t2 = qFar;
  const float t3 = qFar;
  const float D = b * b - 4 * a * cc;
  if (D >= 0) {
    const float q = -0.5f * (b + ssign(b) * sqrtf(D));
    t1 = fabsf(a) > EPS ? q / a : t0;
    t2 = fabsf(q) > EPS ? cc / q : qFar;
    const float min_t = smin(t1, t2);
    t2 = smax(t1, t2);
    t1 = min_t;
    t1 = sclamp(t1, t0, t3);
    t2 = sclamp(t2, t0, t3);
  }
  const bool s0 = c0 > 0;
  const bool s1 = (c0 + t1 * (c1 + t1 * (c2 + t1 * c3))) > 0;
  const bool s2 = (c0 + t2 * (c1 + t2 * (c2 + t2 * c3))) > 0;
  const bool s3 = (c0 + t3 * (c1 + t3 * (c2 + t3 * c3))) > 0;
  float nwt_min = t0, nwt_max = t0;
  if (s0 != s1) {
    nwt_min = t0;
    nwt_max = t1;
  } else if (s1 != s2) {
    nwt_min = t1;
    nwt_max = t2;
  } else if (s2 != s3) {
    nwt_min = t2;
    nwt_max = t3;
  }
  if (!(nwt_min < nwt_max)) return false;
  unsigned nwt_iter = 0;
  float rtn = 0.5f * (nwt_min + nwt_max);
  float f = 1000;
  while (nwt_iter < 10 && fabsf(f) >= EPS) {
    f = c0 + rtn * (c1 + rtn * (c2 + rtn * c3));
    const float df = c1 + rtn * (2 * c2 + rtn * 3 * c3);
    const float dx = f / (df + ssign(df) * 1e-9f);
    rtn -= dx;
    nwt_iter++;
  }
  t = rtn;
  return rtn >= 0 && rtn <= qFar && fabsf(f) < EPS;
}

template <class CTX>
__device__ void local_surface(CTX& c, uint32_t type, f3 ray_dir, uint32_t instId, uint32_t geomId,
                              const float* values, uint32_t primId, float d, float qNear, float qFar, f2 fNearFar,
                              f3 start_q, lrt_hit& hit)
{
  const DevScene& S = c.S;
  const float EPS = 1e-6f;
  const float d_inv = 1.0f / d;
  float t = qNear;
  bool early_hit = false, hitf = false;
  unsigned iter = 0;
  float start_sign = 1;
  float start_dist = trilinear(values, start_q + t * ray_dir);
  c.inc(kCntStSteps);
  if (S.flags & kFlagSurfaceMode) start_sign = ssign(start_dist);
  start_dist *= start_sign;
  const uint32_t solver = CTX::kSolvers ? (S.flags >> kFlagSolverShift) & 7u : kSolverST;
  if (start_dist <= EPS || (S.flags & kFlagBBoxMode)) {
    early_hit = true;
    hitf = true;
  } else if (solver == kSolverST) {
    float dist = start_dist;
    while (t < qFar && dist > EPS && iter < 256) {
      t += dist * d_inv;
      dist = start_sign * trilinear(values, start_q + t * ray_dir);
      iter++;
    }
    c.inc(kCntStSteps, iter);
    hitf = (dist <= EPS);
  } else {
    float cf[4];
    sdf_cubic(values, d_inv, start_q, ray_dir, cf);
    if (solver == kSolverAnalytic) {
      t = sdf_root_analytic(cf, EPS);
      hitf = (t >= 0 && t <= qFar);
    } else if (solver == kSolverNewton) {
      hitf = sdf_root_newton(cf, qFar, EPS, t);
    } else { // IT: interval tracing bounded by the cubic's derivative (:588-618)
      const float c1 = cf[1], c2 = cf[2], c3 = cf[3];
      const float k = 2;
      float e = 0.1f * qFar;
      const float t_max = fabsf(c3) < EPS ? 1e6f : -c2 / (3 * c3);
      const float df_max = 3 * c3 * t_max * t_max + 2 * c2 * t_max + c1;
      float dist = start_dist;
      while (t < qFar && dist > EPS && iter < 256) {
        const float df_1 = 3 * c3 * t * t + 2 * c2 * t + c1;
        const float df_2 = 3 * c3 * (t + e) * (t + e) + 2 * c2 * (t + e) + c1;
        float L = (t_max > t && t_max < t + e) ? smax(df_max, smax(df_1, df_2)) : smax(df_1, df_2);
        L = smax(L, EPS);
        const float st = smin((dist * d_inv) / L, e);
        t += st;
        e = k * st;
        dist = start_sign * trilinear(values, start_q + t * ray_dir);
        iter++;
      }
      c.inc(kCntStSteps, iter);
      hitf = (dist <= EPS);
    }
  }
  const float tReal = fNearFar.x + d * t;
  if (t <= qFar && hitf && tReal < hit.t) {
    // The normal is evaluated once the traversal has ended (trace_one), from
    // what it depends on, kept here: lanes whose hits are found in different
    // iterations of the surrounding loops then compute their normals together.
    f2 en = encode_normal(mk3(0, 0, 1));
    if (S.flags & kFlagNeedNormal) {
      const uint32_t st = blockDim.x;
      // the sample point: start_q itself for the BBOX mode's early hits
      const f3 q = (S.flags & kFlagBBoxMode) ? start_q : start_q + t * ray_dir;
      c.nrec[0] = start_sign;
      c.nrec[st] = q.x;
      c.nrec[2 * st] = q.y;
      c.nrec[3 * st] = q.z;
#pragma unroll
      for (int i = 0; i < 8; i++) c.nrec[(4 + i) * st] = values[i];
      en = mk2(0.0f, 0.0f);
      c.inc(kCntNormals);
    }
    if (CTX::kRecord) {
      c.rec.t = tReal;
#pragma unroll
      for (int i = 0; i < 8; i++) c.rec.values[i] = values[i];
      c.rec.p = start_q + t * ray_dir;
      c.rec.dir = ray_dir;
      c.rec.d = d;
      c.rec.sbs = false; // octree_brick marks its own hits
      c.rec.early = early_hit;
    }
    hit.t = tReal;
    hit.primId = (S.flags & kFlagStIterations) ? iter : primId;
    hit.instId = instId;
    hit.geomId = geomId | (type << 24);
    hit.coords[0] = 0;
    hit.coords[1] = 0;
    hit.coords[2] = en.x;
    hit.coords[3] = en.y;
  }
}

template <class CTX>
__device__ void octree_node(CTX& c, const DevGeom& g, f3 ray_pos, f3 ray_dir, f3 inv_dir, float tNear,
                            uint32_t instId, uint32_t geomId, uint32_t bvhNodeId, lrt_hit& hit)
{
  const DevScene& S = c.S;
  float values[8];
  uint32_t primId;
  f3 min_pos, max_pos;
  if (g.type == LRT_TYPE_SDF_FRAME_OCTREE) {
    c.inc(kCntOctreeLeaves);
    // origNodes box (32 B) + the node's 8 corner values
    const float4* on = reinterpret_cast<const float4*>(S.origNodes + bvhNodeId);
    const float4 a = __ldg(on), b = __ldg(on + 1);
    primId = __float_as_uint(a.w);
    const uint64_t nodeId = uint64_t(primId) + g.sdfRoot;
    min_pos = ld3(a);
    max_pos = ld3(b);
    const float* vals = S.frameOctreeNodes[nodeId].values;
#pragma unroll
    for (int i = 0; i < 8; i++) values[i] = __ldg(vals + i);
  } else {
    c.inc(kCntSvsLeaves);
    primId = bvhNodeId;
    const uint4 n = __ldg(reinterpret_cast<const uint4*>(S.svsNodes) + (uint64_t(primId) + g.sdfRoot));
    const float px = float(n.x >> 16), py = float(n.x & 0x0000FFFF);
    const float pz = float(n.y >> 16), sz = float(n.y & 0x0000FFFF);
    const float d_max = 2 * 1.73205081f / sz;
    min_pos = mk3(-1, -1, -1) + (2.0f * mk3(px, py, pz)) / sz;
    max_pos = min_pos + (2.0f * mk3(1, 1, 1)) / sz;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t w = (i < 4) ? n.z : n.w;
      values[i] = -d_max + 2.0f * d_max * (1.0f / 255.0f) * ((w >> (8 * (i % 4))) & 0xFF);
    }
  }
  const f3 size = max_pos - min_pos;
  const f2 fNearFar = ray_box(ray_pos, inv_dir, min_pos, max_pos); // inv_dir = SafeInverse(ray_dir)
  const f3 start_pos = ray_pos + fNearFar.x * ray_dir;
  const float d = smax(size.x, smax(size.y, size.z));
  const f3 start_q = (start_pos - min_pos) / d;
  const float qFar = (fNearFar.y - fNearFar.x) / d;
  const float qNear = tNear > fNearFar.x ? (tNear - fNearFar.x) / d : 0.0f;
  if (qNear > 0.0f) return; // ray starts inside this node (BVH2Common.cpp:744-745)
  local_surface(c, g.type, ray_dir, instId, geomId, values, primId, d, qNear, qFar, fNearFar, start_q, hit);
}

// FAST: the ray's origin, direction and inverse are finite, so the brick
// and voxel boxes (finite) give no NaN slab value and the one-instruction
// min/max form may be used: a voxel's entry distance is only read when it
// exceeds tNear >= 0.01 (a nonzero value, the same in both forms), and the
// march advance smax(0, far - t) + 1e-6 and the clamped voxel coordinates
// do not depend on the sign of a zero, so every hit is unchanged.
template <bool FAST, class CTX>
__device__ void octree_brick(CTX& c, const DevGeom& g, f3 ray_pos, f3 ray_dir, f3 inv_dir, float tNear,
                             uint32_t instId, uint32_t geomId, uint32_t bvhNodeId, lrt_hit& hit)
{
  const DevScene& S = c.S;
  const DevSbs& sb = S.sbs[g.sdfId];
  const uint32_t primId = bvhNodeId;
  const uint32_t nodeId = primId + g.sdfRoot;
  c.inc(kCntBricks);
  if (primId >= sb.nodeCount) return; // padding box of a one-brick model
  // No voxel of this brick passes the reference's `vmin <= 0` test: its
  // march could only advance t and cannot change the hit.
  const uint32_t* mask = S.sbsMask + sb.maskBase + uint64_t(primId) * sb.maskStride;
  if (__ldg(mask) == 0) return;
  const uint4 node = __ldg(reinterpret_cast<const uint4*>(S.sbsNodes) + nodeId);
  const float px = float(node.x >> 16), py = float(node.x & 0x0000FFFF);
  const float pz = float(node.y >> 16), sz = float(node.y & 0x0000FFFF);
  const uint32_t bs = sb.brick_size;
  const float sz_inv = 2.0f / sz;
  const float d = 2.0f / (sz * bs);
  const f3 brick_min_pos = mk3(-1, -1, -1) + sz_inv * mk3(px, py, pz);
  const f3 brick_max_pos = brick_min_pos + sz_inv * mk3(1, 1, 1);
  const Slabs bsl = slabs(ray_pos, inv_dir, brick_min_pos, brick_max_pos); // inv_dir = SafeInverse(ray_dir)
  f2 bnf = mk2(slab_near<FAST>(bsl), slab_far<FAST>(bsl));
  const float old_t = hit.t;
  const float scale = 0.5f * sz * bs;
  const float hiClamp = bs - 1e-6f;
  const uint32_t V1 = bs + 1;
  const float* dense = S.sbsDense + sb.denseBase + uint64_t(primId) * sb.denseStride;
  float values[8];
  uint32_t steps = 0;
  while (bnf.x < bnf.y && hit.t == old_t) {
    if (steps++ >= S.voxelStepCap) {
      c.err |= kErrVoxelCap;
      break;
    }
    c.inc(kCntVoxels);
    const f3 hit_pos = ray_pos + bnf.x * ray_dir;
    const f3 local_pos = (hit_pos - brick_min_pos) * scale;
    const f3 voxelPos = mk3(floorf(sclamp_pos(local_pos.x, 1e-6f, hiClamp)),
                            floorf(sclamp_pos(local_pos.y, 1e-6f, hiClamp)),
                            floorf(sclamp_pos(local_pos.z, 1e-6f, hiClamp)));
    const f3 min_pos = brick_min_pos + d * voxelPos;
    const f3 max_pos = min_pos + d * mk3(1, 1, 1);
    const uint32_t vx = uint32_t(voxelPos.x), vy = uint32_t(voxelPos.y), vz = uint32_t(voxelPos.z);
    const uint32_t vid = (vx * bs + vy) * bs + vz;
    // surface bit == (min of the 8 corner values <= 0), precomputed
    const bool surface = (__ldg(mask + 1 + (vid >> 5)) >> (vid & 31)) & 1u;
    // the voxel's exit always (for the advance), its entry only where a
    // sphere trace may start
    const Slabs vsl = slabs(ray_pos, inv_dir, min_pos, max_pos);
    const float vfar = slab_far<FAST>(vsl);
    if (surface && tNear < slab_near<FAST>(vsl)) {
      const f2 fNearFar = mk2(slab_near<FAST>(vsl), vfar);
      c.inc(kCntVoxelLoads);
      // 8 corners of the voxel from the dense (bs+1)^3 grid, x-major
      const float* base = dense + (vx * V1 + vy) * V1 + vz;
      values[0] = __ldg(base);
      values[1] = __ldg(base + 1);
      values[2] = __ldg(base + V1);
      values[3] = __ldg(base + V1 + 1);
      values[4] = __ldg(base + V1 * V1);
      values[5] = __ldg(base + V1 * V1 + 1);
      values[6] = __ldg(base + V1 * V1 + V1);
      values[7] = __ldg(base + V1 * V1 + V1 + 1);
      const f3 start_pos = ray_pos + fNearFar.x * ray_dir;
      const f3 start_q = (start_pos - min_pos) * scale;
      const float qFar = (fNearFar.y - fNearFar.x) * scale;
      local_surface(c, g.type, ray_dir, instId, geomId, values, primId, d, 0.0f, qFar, fNearFar, start_q, hit);
      if (CTX::kRecord && hit.t < old_t && sb.colorLayout) {
        // indices of the 8 corner values in the float array (indexed layouts)
        const uint32_t V = sb.vsize, P = sb.pad;
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const uint32_t vId = ((vx + ((i & 4) >> 2) + P) * V + (vy + ((i & 2) >> 1) + P)) * V + (vz + (i & 1) + P);
          c.rec.idx[i] = __ldg(S.sbsData + node.z + vId);
        }
        c.rec.sbs = true;
      }
    }
    bnf.x += smax(0.0f, vfar - bnf.x) + 1e-6f;
  }
  if (hit.t < old_t && sb.colorLayout) {
    // The colour of the hit (indexed layouts) is evaluated once the traversal
    // has ended (trace_one, sbs_hit_colour) from the hit point and the brick,
    // kept here, so that lanes whose hits come in different iterations of the
    // traversal compute their colours together.
    const f3 pos = ray_pos + hit.t * ray_dir;
    const uint32_t st = blockDim.x;
    float* w = c.nrec + kColourWord * st;
    w[0] = pos.x;
    w[st] = pos.y;
    w[2 * st] = pos.z;
    w[3 * st] = __uint_as_float(nodeId);
  }
}

// The hit colour of OctreeBrickIntersect for the indexed layouts
// (BVH2Common.cpp:1081-1110) from the object-space hit point and the brick's
// node, with the brick box computed as octree_brick computes it.
template <class CTX>
__device__ __forceinline__ void sbs_hit_colour(CTX& c, const DevSbs& sb, lrt_hit& hit)
{
  const DevScene& S = c.S;
  const uint32_t st = blockDim.x;
  const float* w = c.nrec + kColourWord * st;
  const f3 pos = mk3(w[0], w[st], w[2 * st]);
  const uint32_t nodeId = __float_as_uint(w[3 * st]);
  const uint4 node = __ldg(reinterpret_cast<const uint4*>(S.sbsNodes) + nodeId);
  const float px = float(node.x >> 16), py = float(node.x & 0x0000FFFF);
  const float pz = float(node.y >> 16), sz = float(node.y & 0x0000FFFF);
  const float sz_inv = 2.0f / sz;
  const f3 brick_min_pos = mk3(-1, -1, -1) + sz_inv * mk3(px, py, pz);
  const f3 dp = (pos - brick_min_pos) * (0.5f * sz);
  const uint32_t* tofs = S.sbsData + node.z + sb.v3;
  f3 col = mk3(0, 0, 0);
#pragma unroll
  for (int k = 0; k < 8; k++) {
    const uint32_t b = __ldg(tofs + k);
    const float wx = (k & 4) ? dp.x : (1 - dp.x);
    const float wy = (k & 2) ? dp.y : (1 - dp.y);
    const float wz = (k & 1) ? dp.z : (1 - dp.z);
    const float wt = wx * wy * wz;
    const f3 cc = wt * mk3(__ldg(S.sbsDataF + b), __ldg(S.sbsDataF + b + 1), __ldg(S.sbsDataF + b + 2));
    col = (k == 0) ? cc : col + cc;
  }
  col = mk3(sclamp(floorf(255.0f * col.x + 0.5f), 0.0f, 255.0f), sclamp(floorf(255.0f * col.y + 0.5f), 0.0f, 255.0f),
            sclamp(floorf(255.0f * col.z + 0.5f), 0.0f, 255.0f));
  hit.coords[0] = col.x + col.y / 256.0f;
  hit.coords[1] = col.z;
}

template <class CTX>
__device__ void triangles(CTX& c, const DevGeom& g, f3 ray_pos, f3 ray_dir, float tNear, uint32_t instId,
                          uint32_t geomId, uint32_t a_start, uint32_t a_count, lrt_hit& hit)
{
  const DevScene& S = c.S;
  const float4* tri = S.triSoup + 3 * (uint64_t(g.triBase) + a_start);
  for (uint32_t i = 0; i < a_count; i++, tri += 3) {
    c.inc(kCntTriTests);
    const float4 A = __ldg(tri), E1 = __ldg(tri + 1), E2 = __ldg(tri + 2);
    const f3 Ap = ld3(A), edge1 = ld3(E1), edge2 = ld3(E2);
    const f3 pvec = cross(ray_dir, edge2);
    const f3 tvec = ray_pos - Ap;
    const f3 qvec = cross(tvec, edge1);
    const float invDet = 1.0f / dot(edge1, pvec);
    const float v = dot(tvec, pvec) * invDet;
    const float u = dot(qvec, ray_dir) * invDet;
    const float t = dot(edge2, qvec) * invDet;
    if (v >= -1e-6f && u >= -1e-6f && (u + v <= 1.0f + 1e-6f) && t > tNear && t < hit.t) {
      hit.t = t;
      hit.primId = a_start + i;
      hit.instId = instId;
      hit.geomId = geomId | (LRT_TYPE_MESH_TRIANGLE << 24);
      hit.coords[0] = u;
      hit.coords[1] = v;
      // the geometric normal is computed once the traversal has ended
      // (trace_one, triangle_normal), from the triangle the hit names
      hit.coords[2] = 0;
      hit.coords[3] = 0;
    }
  }
}

// The normal IntersectAllTrianglesInLeaf writes (BVH2Common.cpp:1609-1625):
// cross(edge1, edge2) of the hit triangle (its triSoup record), through the
// instance's transformInvTransposed, normalised and octahedrally encoded.
__device__ __forceinline__ f2 triangle_normal(const DevScene& S, const DevGeom& g, uint32_t localPrim, uint32_t instId)
{
  const float4* tri = S.triSoup + 3 * (uint64_t(g.triBase) + localPrim);
  const f3 n = cross(ld3(__ldg(tri + 1)), ld3(__ldg(tri + 2)));
  return encode_normal(normalize(matmul4(S.instances[instId].transformInvTransposed, n, 1.0f)));
}

// IntersectAllPrimitivesInLeaf: returns the tag if the hit moved closer.
// inv = SafeInverse(ray_dir); fast: the ray qualifies for the one-instruction
// box tests (fast_nodes).
template <class CTX>
__device__ __forceinline__ uint32_t leaf(CTX& c, const DevGeom& g, f3 ray_pos, f3 ray_dir, f3 inv, bool fast,
                                         float tNear, uint32_t aabbId, uint32_t instId, uint32_t geomId,
                                         lrt_hit& hit)
{
  const float tPrev = hit.t;
  c.inc(kCntLeafCalls);
  const uint32_t packed = __ldg(c.S.primIdCount + g.aabbBase + aabbId);
  const uint32_t a_start = packed & 0x0FFFFFFFu;
  const uint32_t a_count = (packed & 0x70000000u) >> 28;
  switch (g.tag) {
    case LRT_TAG_TRIANGLE: triangles(c, g, ray_pos, ray_dir, tNear, instId, geomId, a_start, a_count, hit); break;
    case LRT_TAG_SDF_NODE: octree_node(c, g, ray_pos, ray_dir, inv, tNear, instId, geomId, a_start, hit); break;
    case LRT_TAG_SDF_BRICK:
      if (fast)
        octree_brick<true>(c, g, ray_pos, ray_dir, inv, tNear, instId, geomId, a_start, hit);
      else
        octree_brick<false>(c, g, ray_pos, ray_dir, inv, tNear, instId, geomId, a_start, hit);
      break;
    default: break;
  }
  return (hit.t >= tPrev) ? LRT_TAG_NONE : g.tag;
}

// Node box test: the literal RayBoxIntersection2 or, when the caller has
// established the conditions under which it decides the same, ray_box_nodes.
template <bool FAST>
__device__ __forceinline__ f2 node_box(f3 o, f3 inv, f3 bmin, f3 bmax)
{
  return FAST ? ray_box_nodes(o, inv, bmin, bmax) : ray_box(o, inv, bmin, bmax);
}

// Rays for which ray_box_nodes decides every node test like ray_box: finite
// origin and direction (so a finite, non-zero inverse never meets an
// infinite difference) and finite inverse, in a scene whose boxes are clean.
__device__ __forceinline__ bool fast_nodes(const DevScene& S, f3 o, f3 d, f3 inv)
{
  return (S.flags & kFlagCleanBoxes) && finite3(o) && finite3(d) && finite3(inv);
}

// The descent of BVH2TraverseF32 (BVH2Common.cpp:3256-3284) down to the next
// leaf; false if the stack would overflow.
template <bool FAST, class CTX>
__device__ __forceinline__ bool blas_descend(CTX& c, const float4* pairs, uint32_t* stack, uint32_t stride,
                                             uint32_t cap, f3 ray_pos, f3 inv, float tNear, float tHit, int& top,
                                             uint32_t& leftNodeOffset)
{
  while (top >= 0 && ((leftNodeOffset & kLeafBit) == 0)) {
    c.inc(kCntBlasPairs);
    const float4* p = pairs + 4 * uint64_t(leftNodeOffset);
    const float4 l0 = __ldg(p), l1 = __ldg(p + 1), r0 = __ldg(p + 2), r1 = __ldg(p + 3);
    const uint32_t n0 = __float_as_uint(l0.w), n1 = __float_as_uint(r0.w);
    const f2 tm0 = node_box<FAST>(ray_pos, inv, ld3(l0), ld3(l1));
    const f2 tm1 = node_box<FAST>(ray_pos, inv, ld3(r0), ld3(r1));
    const bool h0 = (tm0.x <= tm0.y) && (tm0.y >= tNear) && (tm0.x <= tHit);
    const bool h1 = (tm1.x <= tm1.y) && (tm1.y >= tNear) && (tm1.x <= tHit);
    leftNodeOffset = h0 ? n0 : n1;
    if (h0 && h1) {
      if (uint32_t(top) >= cap) {
        c.err |= kErrStackOverflow;
        return false;
      }
      const bool nearFirst = tm0.x <= tm1.x;
      leftNodeOffset = nearFirst ? n0 : n1;
      stack[top * stride] = nearFirst ? n1 : n0;
      top++;
    }
    if (!h0 && !h1) {
      top--;
      leftNodeOffset = stack[(top > 0 ? top : 0) * stride];
    }
  }
  return true;
}

// BVH2TraverseF32 with the stack in shared memory (thread-strided).
template <class CTX>
__device__ void blas(CTX& c, uint32_t* stack, uint32_t stride, uint32_t cap, f3 ray_pos, f3 ray_dir,
                     float tNear, uint32_t instId, uint32_t geomId, bool stopOnFirstHit, lrt_hit& hit)
{
  const DevScene& S = c.S;
  const DevGeom g = S.geoms[geomId];
  const float4* pairs = reinterpret_cast<const float4*>(S.pairs + g.bvhOffset);
  int top = 0;
  uint32_t leftNodeOffset = 0;
  bool hitFound = false;
  stack[0] = 0;
  const f3 inv = safe_inverse(ray_dir);
  const bool fast = fast_nodes(S, ray_pos, ray_dir, inv);
  while (top >= 0 && !hitFound) {
    const bool ok = fast ? blas_descend<true>(c, pairs, stack, stride, cap, ray_pos, inv, tNear, hit.t, top,
                                              leftNodeOffset)
                         : blas_descend<false>(c, pairs, stack, stride, cap, ray_pos, inv, tNear, hit.t, top,
                                               leftNodeOffset);
    if (!ok) return;
    if (top >= 0 && leftNodeOffset != 0xFFFFFFFFu) {
      const float tNearSdf = smax(tNear, 0.01f); // SDF_BIAS (BVH2Common.cpp:3306-3307)
      const uint32_t tag =
          leaf(c, g, ray_pos, ray_dir, inv, fast, tNearSdf, leftNodeOffset & 0x0FFFFFFFu, instId, geomId, hit);
      hitFound = (tag != 0) && (tag != LRT_TAG_TRIANGLE || stopOnFirstHit);
    }
    top--;
    leftNodeOffset = stack[(top > 0 ? top : 0) * stride];
  }
}

// The stackless TLAS walk of RayQuery_NearestHit (BVH2Common.cpp:3346-3358)
// up to the next intersected leaf or the end of the escape chain.
template <bool FAST, class CTX>
__device__ __forceinline__ void tlas_walk(CTX& c, f3 pos, f3 inv, float tmin, float tHit, uint32_t& nodeIdx,
                                          uint32_t& travFlags, uint32_t& leftOffset)
{
  do {
    c.inc(kCntTlasNodes);
    const float4* np = reinterpret_cast<const float4*>(c.S.tlas + nodeIdx);
    const float4 a = __ldg(np), b = __ldg(np + 1);
    const f2 bh = node_box<FAST>(pos, inv, ld3(a), ld3(b));
    const uint32_t intersects = (bh.x <= bh.y) && (bh.y > tmin) && (bh.x < tHit);
    const uint32_t lo = __float_as_uint(a.w);
    travFlags = (lo & kLeafBit) | intersects;
    leftOffset = lo;
    const bool leafOrNot = (travFlags & kLeafBit) != 0 || (travFlags & 1) == 0;
    nodeIdx = leafOrNot ? __float_as_uint(b.w) : leftOffset;
  } while (travFlags != (kLeafBit | 1u) && nodeIdx != 0 && nodeIdx < 0xFFFFFFFEu);
}

// RayQuery_NearestHit for one ray.
template <class CTX>
__device__ void trace_one(CTX& c, uint32_t* stack, uint32_t stride, uint32_t cap, float4 pn, float4 df,
                          lrt_hit& hit)
{
  const DevScene& S = c.S;
  float dirW = df.w;
  const bool stopOnFirstHit = (dirW <= 0.0f);
  if (stopOnFirstHit) dirW *= -1.0f;
  const f3 pos = mk3(pn.x, pn.y, pn.z), dir = mk3(df.x, df.y, df.z);
  const float tmin = pn.w;
  const f3 inv = safe_inverse(dir);
  hit.t = dirW;
  hit.primId = 0xFFFFFFFFu;
  hit.instId = 0xFFFFFFFFu;
  hit.geomId = 0xFFFFFFFFu;
  hit.coords[0] = 1.0f;
  hit.coords[1] = 0.0f;
  hit.coords[2] = 0.0f;
  hit.coords[3] = 0.0f;
  uint32_t nodeIdx = 0;
  const bool fast = fast_nodes(S, pos, dir, inv);
  do {
    uint32_t travFlags = 0, leftOffset = 0;
    if (fast)
      tlas_walk<true>(c, pos, inv, tmin, hit.t, nodeIdx, travFlags, leftOffset);
    else
      tlas_walk<false>(c, pos, inv, tmin, hit.t, nodeIdx, travFlags, leftOffset);
    if (travFlags == (kLeafBit | 1u)) {
      const uint32_t instId = leftOffset & 0x0FFFFFFFu;
      const DevInstance& I = S.instances[instId];
      c.inc(kCntInstances);
      const f3 rp = matmul4(I.transformInv, pos, 1.0f);
      const f3 rd = matmul4(I.transformInv, dir, 0.0f);
      blas(c, stack, stride, cap, rp, rd, tmin, instId, I.geomId, stopOnFirstHit, hit);
      if (c.err & kErrStackOverflow) break;
    }
  } while (nodeIdx < 0xFFFFFFFEu && !(stopOnFirstHit && hit.primId != 0xFFFFFFFFu));
  // What the leaf tests left for the end of the traversal: the final hit's
  // normal, an SBS hit's colour and the triangle primId remap.
  if (hit.geomId < 0xFFFFFFFFu) {
    const DevGeom& g = S.geoms[hit.geomId & 0x00FFFFFFu];
    if ((hit.geomId >> 24) == LRT_TYPE_MESH_TRIANGLE) {
      if (S.flags & kFlagNeedNormal) {
        const f2 en = triangle_normal(S, g, hit.primId, hit.instId);
        hit.coords[2] = en.x;
        hit.coords[3] = en.y;
      }
      c.triLocal = hit.primId;
      hit.primId = __ldg(S.primIndices + g.triBase + hit.primId);
    } else {
      if (S.flags & kFlagNeedNormal) {
        const f2 en = deferred_normal(c, hit.instId);
        hit.coords[2] = en.x;
        hit.coords[3] = en.y;
      }
      if (g.tag == LRT_TAG_SDF_BRICK) {
        const DevSbs& sb = S.sbs[g.sdfId];
        if (sb.colorLayout) sbs_hit_colour(c, sb, hit);
      }
    }
  }
  if (hit.primId != 0xFFFFFFFFu) c.inc(kCntHits);
}

// Longest-first order of the tiles of an image-order launch.  Each launch
// times its tiles on lane 0 and sorts the slow ones into three classes by
// their cost against the previous launch's longest tile (at least 1/2, 1/4,
// 1/8 of it); the next launch of the same image size on the same stream
// (rd) hands out class 0, then 1, then 2, each in the order the tiles
// finished, then every other tile in natural order (a bitmap skips the
// listed ones).  If the previous launch was tail-bound (its longest tile
// took longer than its warps' mean busy time), a class-0 tile goes out as
// kSplitParts work items, each traced by one warp on its own rows of the
// tile; the parts' costs add up in the tile's accumulator and the last part
// to finish records the tile.  Only which warp traces which ray, and when,
// depends on it.
// rd == nullptr: natural order; wr == nullptr: nothing recorded.  Buffer
// layout: sched_words and the offsets beside it (device_layout.h).  The
// per-warp state lives in shared memory so that the traversal keeps its
// registers.
//
// A work item is a tile index with, for the part of a split tile, bit 31 set
// and the part in bits 24..30 (tile counts stay below 2^24).
struct WarpClock {
  long long start;  // clock64 when the warp took its current item
  uint32_t item;    // that item, ~0u before the first
  uint32_t longest; // longest tile this warp has reported
  uint32_t pos;     // a split item's position in the concatenated class lists
  unsigned long long busy; // sum of the costs of the items this warp traced
};
constexpr uint32_t kItemSplit = 0x80000000u;
constexpr uint32_t kItemTileMask = 0x00FFFFFFu;

__device__ __forceinline__ uint32_t item_tile(uint32_t item) { return item & kItemTileMask; }

// Whether `lane` traces its pixel of the item's tile: every lane for a whole
// tile, rows part * (32 / kSplitParts) ... of it for a part.
__device__ __forceinline__ bool item_has_lane(uint32_t item, uint32_t lane)
{
  return !(item & kItemSplit) || lane / (32u / kSplitParts) == ((item >> 24) & 0x7Fu);
}

// lane 0: records that a tile took `cost` (longest, class list, bitmap).
__device__ __forceinline__ void sched_record(const uint32_t* __restrict__ rd, uint32_t* wr, uint32_t tiles,
                                             uint32_t tile, uint32_t cost, WarpClock& wc)
{
  const uint64_t lists = sched_lists_offset(tiles);
  if (cost > wc.longest) {
    wc.longest = cost;
    atomicMax(wr, cost);
  }
  const uint32_t mx = rd ? __ldg(rd) : 0u;
  if (mx) {
    const int cls = cost >= mx / 2 ? 0 : cost >= mx / 4 ? 1 : cost >= mx / 8 ? 2 : 3;
    if (cls < 3) {
      const uint32_t slot = atomicAdd(wr + 1 + cls, 1u);
      if (slot < tiles) wr[lists + cls * tiles + slot] = tile;
      atomicOr(wr + kSchedHeader + (tile >> 5), 1u << (tile & 31));
    }
  }
}

// lane 0, after the warp has finished its current item (if any): records
// that item's duration and returns the next item of `tiles`, ~0u when none
// is left.
__device__ __forceinline__ uint32_t sched_next(const uint32_t* __restrict__ rd, uint32_t* wr, uint32_t tiles,
                                               unsigned long long* counter, WarpClock& wc)
{
  const uint64_t lists = sched_lists_offset(tiles);
  if (wr && wc.item != ~0u) {
    const long long dt = (clock64() - wc.start) >> 4;
    uint32_t cost = uint32_t(dt < 0xFFFFFFFFll ? dt : 0xFFFFFFFFll);
    bool record = true;
    if (wc.item & kItemSplit) { // parts add up; the last one records the tile
      unsigned long long* acc = reinterpret_cast<unsigned long long*>(wr + sched_acc_offset(tiles));
      const unsigned long long prev = atomicAdd(acc + wc.pos, (1ull << 40) | cost);
      record = (prev >> 40) + 1 == kSplitParts;
      const unsigned long long sum = (prev & ((1ull << 40) - 1)) + cost;
      cost = uint32_t(sum < 0xFFFFFFFFull ? sum : 0xFFFFFFFFull);
    }
    wc.busy += cost;
    if (record) sched_record(rd, wr, tiles, item_tile(wc.item), cost, wc);
  }
  static_assert(kSchedClasses == 3, "three cost classes");
  static_assert(kSplitParts >= 1 && kSplitParts <= 32 && (32 % kSplitParts) == 0, "parts of a 32-lane tile");
  uint32_t n[3] = {0, 0, 0};
  if (rd)
    for (int c = 0; c < 3; c++) n[c] = min(__ldg(rd + 1 + c), tiles);
  const uint64_t nAll = uint64_t(n[0]) + n[1] + n[2];
  // class-0 tiles go out in kSplitParts parts if the previous launch was
  // tail-bound: longest * warps > sum of the warps' busy times
  const bool tailBound =
      rd && uint64_t(__ldg(rd)) * __ldg(rd + kSchedWarps) >
                __ldg(reinterpret_cast<const unsigned long long*>(rd + kSchedBusy));
  const uint64_t nSplit = tailBound ? n[0] : 0;
  const uint64_t nItems = nSplit * kSplitParts + (nAll - nSplit);
  for (;;) {
    const unsigned long long k = atomicAdd(counter, 1ull);
    uint32_t item;
    if (k < nItems) {
      const bool split = k < nSplit * kSplitParts;
      const uint64_t j = split ? k / kSplitParts : k - nSplit * (kSplitParts - 1);
      const int cls = j < n[0] ? 0 : j < uint64_t(n[0]) + n[1] ? 1 : 2;
      const uint64_t jj = cls == 0 ? j : cls == 1 ? j - n[0] : j - n[0] - n[1];
      const uint32_t tile = __ldg(rd + lists + cls * tiles + jj);
      if (tile >= tiles) continue;
      item = (split && kSplitParts > 1) ? tile | kItemSplit | (uint32_t(k % kSplitParts) << 24) : tile;
      wc.pos = uint32_t(j);
    } else {
      if (k - nItems >= tiles) { // none left: report this warp's busy time
        if (wr) {
          atomicAdd(reinterpret_cast<unsigned long long*>(wr + kSchedBusy), wc.busy);
          atomicAdd(wr + kSchedWarps, 1u);
        }
        return wc.item = ~0u;
      }
      item = uint32_t(k - nItems);
      if (nAll && ((__ldg(rd + kSchedHeader + (item >> 5)) >> (item & 31)) & 1u)) continue;
    }
    wc.start = clock64();
    return wc.item = item;
  }
}

// One thread per ray; warps fetch 32-ray batches from a global counter
// (persistent grid of ~one wave).  Stacks live in shared memory,
// stack[i * blockDim + tid].
//
// With img_w > 0 the n = img_w * img_h rays form an image in row-major pixel
// order and a warp's 32 rays are an 8x4-pixel tile instead of 32 pixels of a
// row (the reference's kernel1D_FillGbuffer also walks pixels in packed
// tiles, MultiRenderer.cpp:185-202); each ray's hit is unchanged.
// The L2 prefetch of a small scene (DevScene::pfPtr): CTA b of the grid
// takes the b-th share of each range, in whole kPrefetchChunk pieces, and
// its first warp issues one cp.async.bulk.prefetch.L2 per piece (no result,
// no completion to wait for).  Bases are 16-byte aligned and sizes multiples
// of 16, so every piece is too.
__device__ __forceinline__ void l2_prefetch_scene(const DevScene& S)
{
  if (threadIdx.x >= 32) return;
#pragma unroll 1
  for (int r = 0; r < kPrefetchRanges; r++) {
    const uint64_t bytes = S.pfBytes[r];
    if (bytes == 0) continue;
    const uint64_t per = (bytes + gridDim.x - 1) / gridDim.x;
    const uint64_t share = (per + kPrefetchChunk - 1) / kPrefetchChunk * kPrefetchChunk;
    const uint64_t lo = min(bytes, share * blockIdx.x), hi = min(bytes, lo + share);
    for (uint64_t off = lo + uint64_t(threadIdx.x) * kPrefetchChunk; off < hi; off += 32ull * kPrefetchChunk) {
      const uint32_t size = uint32_t(min(uint64_t(kPrefetchChunk), hi - off));
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(S.pfPtr[r] + off), "r"(size) : "memory");
    }
  }
}

//
// MINB: blocks per SM the register allocation is bounded for (7: 72
// registers; 6: 80 registers, used for the image-order launches of scenes
// whose geometries are all sparse-brick sets, where the brick march and the
// sphere trace spill at 72, and for row-order launches smaller than one wave,
// which wait on their slowest warp's chain of dependent steps).
template <bool COUNT, bool SOLVERS, bool IMG, int MINB = 7>
__global__ void __launch_bounds__(kTraceThreads, MINB) k_trace(DevScene S, const float4* __restrict__ rays,
                                                         lrt_hit* __restrict__ hits, uint64_t n,
                                                         unsigned long long* __restrict__ work_counter,
                                                         unsigned long long* __restrict__ counters,
                                                         uint32_t* __restrict__ err_word, uint32_t stack_cap,
                                                         uint32_t img_w, uint32_t img_h,
                                                         const uint32_t* __restrict__ sched_rd, uint32_t* sched_wr,
                                                         uint32_t group)
{
  extern __shared__ uint32_t smem_stack[];
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  Ctx<COUNT, false, SOLVERS> c(S, normal_words(smem_stack, stack_cap));
  __shared__ WarpClock wclock[IMG ? kTraceThreads / 32 : 1];
  const uint64_t tilesX = (uint64_t(img_w) + kImgTileW - 1) / kImgTileW;
  if (IMG && lane == 0) {
    wclock[threadIdx.x >> 5].item = ~0u;
    wclock[threadIdx.x >> 5].longest = 0;
    wclock[threadIdx.x >> 5].busy = 0;
  }
  l2_prefetch_scene(S);
  for (;;) {
    unsigned long long base = 0;
    bool mine = true; // this lane's pixel belongs to the work item
    if (IMG) { // work counter in tiles
      __syncwarp();
      uint32_t item = 0;
      if (lane == 0)
        item = sched_next(sched_rd, sched_wr, uint32_t(tilesX * ((img_h + kImgTileH - 1) / kImgTileH)), work_counter,
                          wclock[threadIdx.x >> 5]);
      item = __shfl_sync(0xFFFFFFFFu, item, 0);
      if (item == ~0u) break;
      base = uint64_t(item_tile(item)) * 32;
      mine = item_has_lane(item, lane);
    } else { // in rays, `group` (32, 16 or 8) to a warp
      if (lane == 0) base = atomicAdd(work_counter, (unsigned long long)group);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base >= n) break;
    }
    uint64_t i = base + lane;
    bool valid = i < n && (IMG || lane < group);
    if (!IMG && group < 32) {
      // A launch smaller than one wave lasts as long as its slowest warp, and
      // the slow rays of an image (grazing ones) lie next to each other: warp
      // g takes rays g, g + G, g + 2G, ... of the G groups instead of `group`
      // consecutive ones, so that they spread over many warps.
      const uint64_t G = (n + group - 1) / group;
      i = base / group + uint64_t(lane) * G;
      valid = lane < group && i < n;
    }
    if (IMG) {
      const uint64_t b = base >> 5;
      const uint32_t x = uint32_t(b % tilesX) * kImgTileW + (lane % kImgTileW);
      const uint32_t y = uint32_t(b / tilesX) * kImgTileH + (lane / kImgTileW);
      valid = x < img_w && y < img_h && mine;
      i = uint64_t(y) * img_w + x;
      valid = valid && i < n; // a row-order launch traced as an 8-wide image has a ragged last row
    }
    if (valid) {
      const float4 pn = __ldg(rays + 2 * i), df = __ldg(rays + 2 * i + 1);
      lrt_hit h;
      trace_one(c, stack, blockDim.x, stack_cap, pn, df, h);
      float4* out = reinterpret_cast<float4*>(hits + i);
      out[0] = make_float4(h.t, __uint_as_float(h.primId), __uint_as_float(h.instId), __uint_as_float(h.geomId));
      out[1] = make_float4(h.coords[0], h.coords[1], h.coords[2], h.coords[3]);
    }
  }
  if (c.err) atomicOr(err_word, c.err);
  if (COUNT) {
#pragma unroll
    for (int k = 0; k < LRT_COUNTER_COUNT; k++) {
      uint32_t v = c.cnt.c[k];
      // warp-reduce before the atomic
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
      if (lane == 0 && v) atomicAdd(counters + k, (unsigned long long)v);
    }
  }
}

// Tonemap (MultiRenderer_resolve.cpp:536-542) of one colour to RGBA8.
__device__ __forceinline__ uint32_t tonemap_rgba8(float r, float g, float b, float a)
{
  // uint4(255 * clamp(color, 0, 1)): clamp as LiteMath's min(max(a, u), b)
  const uint32_t x = uint32_t(255.0f * sclamp(r, 0.0f, 1.0f));
  const uint32_t y = uint32_t(255.0f * sclamp(g, 0.0f, 1.0f));
  const uint32_t z = uint32_t(255.0f * sclamp(b, 0.0f, 1.0f));
  const uint32_t w = uint32_t(255.0f * sclamp(a, 0.0f, 1.0f));
  return (w << 24) | (z << 16) | (y << 8) | x;
}

// ResolveCommon for LAMBERT_NO_TEX (white albedo, the lights of L, the
// background for misses) and Tonemap of one traced eye ray; c.triLocal is
// the triangle record of a triangle hit (set by trace_one).
template <class CTX>
__device__ __forceinline__ uint32_t resolve_rgba8(CTX& c, const DevLights& L, f3 rayPos, f3 rayDir,
                                                  const lrt_hit& h)
{
  const DevScene& S = c.S;
  if (h.primId == 0xFFFFFFFFu) {
    return tonemap_rgba8(L.background[0], L.background[1], L.background[2], L.background[3]);
  } else {
    f3 norm;
    if ((h.geomId >> 24) == LRT_TYPE_MESH_TRIANGLE) {
      const DevGeom& g = S.geoms[h.geomId & 0x00FFFFFFu];
      const float4* tri = S.triSoup + 3 * (uint64_t(g.triBase) + c.triLocal);
      const f3 raw = cross(ld3(__ldg(tri + 1)), ld3(__ldg(tri + 2)));
      norm = normalize(matmul4(S.instances[h.instId].transformInvTransposed, raw, 1.0f));
      norm = ssign(dot(-1.0f * rayDir, norm)) * norm;
    } else {
      norm = decode_normal(mk2(h.coords[2], h.coords[3]));
    }
    const f3 color = mk3(1, 1, 1);
    f3 fc = mk3(0, 0, 0);
    for (uint32_t i = 0; i < L.count; i++) {
      const DevLight& l = L.light[i];
      const f3 lc = mk3(l.color[0], l.color[1], l.color[2]);
      const f3 sp = mk3(l.space[0], l.space[1], l.space[2]);
      if (l.type == LRT_LIGHT_DIRECT) {
        const float q = smax(0.0f, dot(norm, sp));
        fc = fc + (lc * color) * q;
      } else if (l.type == LRT_LIGHT_POINT) {
        const f3 surf = rayPos + h.t * rayDir;
        f3 dir = sp - surf;
        const float len = sqrtf(dot(dir, dir));
        dir = mk3(dir.x / len, dir.y / len, dir.z / len);
        const float q = smax(0.0f, dot(norm, dir));
        fc = fc + ((lc * color) * q) / (len * len);
      } else {
        fc = fc + lc * color;
      }
    }
    return tonemap_rgba8(fc.x, fc.y, fc.z, 1.0f);
  }
}

// MultiRenderer::AnyHit (MultiRenderer.cpp:223-246) for the eye ray r:
// nearest hits composited front to back, each trace restarting at the
// previous hit point with r's tNear and direction, until the remaining alpha
// is at most 0.01 or, unlike the reference's loop, after
// LRT_MAX_TRANSPARENCY_LAYERS traces (error bit).  Misses take the
// background; SBS_COL (11) and graphics-primitive (17) hits keep the
// previous colour.  h is the last hit; tc and alpha the composited colour
// and the remaining alpha.
template <class CTX>
__device__ void anyhit_loop(CTX& c, uint32_t* stack, uint32_t stack_cap, const DevMaterials& M, const float* r,
                            lrt_hit& h, f3& tc, float& alpha)
{
  f3 pos = mk3(r[0], r[1], r[2]);
  const f3 dir = mk3(r[4], r[5], r[6]);
  tc = mk3(0.0f, 0.0f, 0.0f);
  alpha = 1.0f;
  float4 color = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (uint32_t layer = 0;; layer++) {
    if (layer == LRT_MAX_TRANSPARENCY_LAYERS) {
      c.err |= kErrLayerCap;
      break;
    }
    const float wa = alpha * color.w;
    tc = mk3(tc.x + wa * color.x, tc.y + wa * color.y, tc.z + wa * color.z);
    alpha *= (1.0f - color.w);
    trace_one(c, stack, blockDim.x, stack_cap, make_float4(pos.x, pos.y, pos.z, r[3]),
              make_float4(r[4], r[5], r[6], r[7]), h);
    const uint32_t type = h.geomId >> 24, geomId = h.geomId & 0x00FFFFFFu;
    if (h.primId == 0xFFFFFFFFu) {
      color = make_float4(M.background[0], M.background[1], M.background[2], M.background[3]);
    } else if (type != LRT_TYPE_SDF_SBS_COL && type != LRT_TYPE_GRAPHICS_PRIM) {
      const uint2 o = M.offsets[geomId];
      const lrt_material& m = M.mats[M.ids[o.x + h.primId % o.y]];
      color = m.type == LRT_MATERIAL_COLORED
                  ? make_float4(m.base_color[0], m.base_color[1], m.base_color[2], m.base_color[3])
                  : make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    }
    pos = pos + h.t * dir;
    if (!(alpha > 0.01f)) break;
  }
}

// MultiRenderer's colour palettes (MultiRenderer.h:269-283): objects by id
// and LOD levels, RGBA8 words.
__constant__ uint32_t kPalette[20] = {0xffe6194b, 0xff3cb44b, 0xffffe119, 0xff0082c8, 0xfff58231,
                                      0xff911eb4, 0xff46f0f0, 0xfff032e6, 0xffd2f53c, 0xfffabebe,
                                      0xff008080, 0xffe6beff, 0xffaa6e28, 0xfffffac8, 0xff800000,
                                      0xffaaffc3, 0xff808000, 0xffffd8b1, 0xff000080, 0xff808080};
__constant__ uint32_t kLodPalette[20] = {0xff000000, 0xff000040, 0xff000080, 0xff0000c0, 0xff0040ff,
                                         0xff0080ff, 0xff00c0ff, 0xff00ffff, 0xff00ffc0, 0xff00ff80,
                                         0xff00ff40, 0xff00ff00, 0xff00c000, 0xff008000, 0xff004000,
                                         0xff000000, 0xffff0000, 0xffff0000, 0xffff0000, 0xffff0000};

// decode_RGBA8 (utils/raytracing/render_common.h:250-254)
__device__ __forceinline__ float4 decode_rgba8(uint32_t c)
{
  return make_float4(float(c & 0xFF) * (1.0f / 255.0f), float((c >> 8) & 0xFF) * (1.0f / 255.0f),
                     float((c >> 16) & 0xFF) * (1.0f / 255.0f), float((c >> 24) & 0xFF) * (1.0f / 255.0f));
}

// The colour of SBS_COL and graphics-primitive hits packed in coords[0..1]
// (MultiRenderer_resolve.cpp:629-634): round / 255, the fraction, round / 255.
__device__ __forceinline__ f3 packed_hit_colour(const lrt_hit& h)
{
  return mk3(roundf(h.coords[0]) / 255.0f, h.coords[0] - floorf(h.coords[0]), roundf(h.coords[1]) / 255.0f);
}

// Sum of the lights' Lambert terms for base colour `color` (ResolveCommon,
// MultiRenderer_resolve.cpp:638-663).
__device__ __forceinline__ f3 lambert_lights(const DevLights& L, f3 norm, f3 color, f3 rayPos, f3 rayDir, float t)
{
  f3 fc = mk3(0, 0, 0);
  for (uint32_t i = 0; i < L.count; i++) {
    const DevLight& l = L.light[i];
    const f3 lc = mk3(l.color[0], l.color[1], l.color[2]);
    const f3 sp = mk3(l.space[0], l.space[1], l.space[2]);
    if (l.type == LRT_LIGHT_DIRECT) {
      const float q = smax(0.0f, dot(norm, sp));
      fc = fc + (lc * color) * q;
    } else if (l.type == LRT_LIGHT_POINT) {
      const f3 surf = rayPos + t * rayDir;
      f3 dir = sp - surf;
      const float len = sqrtf(dot(dir, dir));
      dir = mk3(dir.x / len, dir.y / len, dir.z / len);
      const float q = smax(0.0f, dot(norm, dir));
      fc = fc + ((lc * color) * q) / (len * len);
    } else {
      fc = fc + lc * color;
    }
  }
  return fc;
}

// ResolveCommon / kernel1D_ResolveDebug (MultiRenderer_resolve.cpp:580-666,
// 810-990) of one traced eye ray for the render modes without textures,
// shadows or PBR, before Tonemap (alpha 1 for hits, the background's for
// misses): MASK, DEPTH, LINEAR_DEPTH,
// INVERSE_LINEAR_DEPTH, PRIMITIVE, TYPE, GEOM, NORMAL, BARYCENTRIC,
// ST_ITERATIONS, DIFFUSE, LAMBERT, HSV_DEPTH, LOD, MATERIAL, MO_VOXEL_COUNT
// and MO_FLAGS (colored materials only).  The normal is loadNormalTcFromGbuffer's
// (triangles recomputed and turned to the viewer, SDF hits decoded).
// Image2D<float4>::sample (dependencies/1st-party/LiteMath/Image2d.cpp:
// 105-183) with the sampler every MultiRenderer texture has (AddTexture,
// MultiRenderer_host.cpp:827-839): LINEAR filter, CLAMP addressing
// (bilinearOffsets, Image2d.cpp:50-102), in its operation order.
__device__ __forceinline__ float4 sample_texture(const DevMaterials& M, uint32_t tex, float u, float v)
{
  if (tex >= M.texCount) return make_float4(0, 0, 0, 0);
  const uint4 t = __ldg(M.texs + tex);
  const int w = int(t.y), hgt = int(t.z);
  const float4* data = M.texels + t.x;
  float ffx = u * float(w) - 0.5f;
  float ffy = v * float(hgt) - 0.5f;
  if (ffx < 0) ffx = 0.0f;
  if (ffy < 0) ffy = 0.0f;
  const int px = int(ffx), py = int(ffy);
  const float fx = fabsf(ffx - float(px)), fy = fabsf(ffy - float(py));
  const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
  const float w1 = fx1 * fy1, w2 = fx * fy1, w3 = fx1 * fy, w4 = fx * fy;
  int px0 = px >= w ? w - 1 : px, px1 = px + 1 >= w ? w - 1 : px + 1;
  int py0 = py >= hgt ? hgt - 1 : py, py1 = py + 1 >= hgt ? hgt - 1 : py + 1;
  px0 = px0 < 0 ? 0 : px0;
  px1 = px1 < 0 ? 0 : px1;
  py0 = py0 < 0 ? 0 : py0;
  py1 = py1 < 0 ? 0 : py1;
  const float4 f1 = __ldg(data + int64_t(py0) * w + px0), f2 = __ldg(data + int64_t(py0) * w + px1);
  const float4 f3 = __ldg(data + int64_t(py1) * w + px0), f4 = __ldg(data + int64_t(py1) * w + px1);
  return make_float4(f1.x * w1 + f2.x * w2 + f3.x * w3 + f4.x * w4, f1.y * w1 + f2.y * w2 + f3.y * w3 + f4.y * w4,
                     f1.z * w1 + f2.z * w2 + f3.z * w3 + f4.z * w4, f1.w * w1 + f2.w * w2 + f3.w * w3 + f4.w * w4);
}

template <class CTX>
__device__ float4 resolve_mode_colour(CTX& c, const DevLights& L, const DevMaterials& M, uint32_t mode, f3 rayPos,
                                      f3 rayDir, const lrt_hit& h)
{
  const DevScene& S = c.S;
  if (h.primId == 0xFFFFFFFFu) return make_float4(L.background[0], L.background[1], L.background[2], L.background[3]);
  const uint32_t type = h.geomId >> 24, geomId = h.geomId & 0x00FFFFFFu;
  f3 norm;
  // loadNormalTcFromGbuffer's texture coordinates (:27-76): SDF hits' coords[0..1]
  float tcu = h.coords[0], tcv = h.coords[1];
  if (type == LRT_TYPE_MESH_TRIANGLE) {
    const DevGeom& g = S.geoms[geomId];
    const uint64_t slot = uint64_t(g.triBase) + c.triLocal;
    const float4* tri = S.triSoup + 3 * slot;
    const f3 raw = cross(ld3(__ldg(tri + 1)), ld3(__ldg(tri + 2)));
    norm = normalize(matmul4(S.instances[h.instId].transformInvTransposed, raw, 1.0f));
    norm = ssign(dot(-1.0f * rayDir, norm)) * norm;
    // (1 - c0 - c1) * A_tc + c1 * B_tc + c0 * C_tc of the vertices' coordinates
    float2 A = make_float2(0, 0), B = A, C = A;
    if (M.triTc) {
      A = __ldg(M.triTc + 3 * slot);
      B = __ldg(M.triTc + 3 * slot + 1);
      C = __ldg(M.triTc + 3 * slot + 2);
    }
    const float wa = 1.0f - h.coords[0] - h.coords[1];
    tcu = wa * A.x + h.coords[1] * B.x + h.coords[0] * C.x;
    tcv = wa * A.y + h.coords[1] * B.y + h.coords[0] * C.y;
  } else {
    norm = decode_normal(mk2(h.coords[2], h.coords[3]));
  }
  auto material = [&]() -> const lrt_material& {
    const uint2 o = M.offsets[geomId];
    return M.mats[M.ids[o.x + h.primId % o.y]];
  };
  // a material's colour: base_color if COLORED, else its texture at the hit's coordinates
  auto material_colour = [&](const lrt_material& m) -> float4 {
    if (m.type == LRT_MATERIAL_COLORED) return make_float4(m.base_color[0], m.base_color[1], m.base_color[2],
                                                           m.base_color[3]);
    return sample_texture(M, m.texId, tcu, tcv);
  };
  const float z = h.t, z_near = 0.1f, z_far = 10.0f;
  float4 res = make_float4(1, 0, 1, 1);
  switch (mode) {
  case 0: // MASK
    res = make_float4(1, 1, 1, 1);
    break;
  case 2: { // DEPTH
    const float d = (1.0f / z - 1.0f / z_near) / (1.0f / z_far - 1.0f / z_near);
    res = make_float4(d, d, d, 1);
  } break;
  case 3: { // LINEAR_DEPTH
    const float d = (z - z_near) / (z_far - z_near);
    res = make_float4(d, d, d, 1);
  } break;
  case 4: { // INVERSE_LINEAR_DEPTH
    const float d = 1 - ((z - z_near) / (z_far - z_near));
    res = make_float4(d, d, d, 1);
  } break;
  case 5: // PRIMITIVE
  case 25: // MO_FLAGS
    res = decode_rgba8(kPalette[h.primId % 20]);
    break;
  case 6: // TYPE
    res = decode_rgba8(kPalette[type % 20]);
    break;
  case 22: // MATERIAL
    res = decode_rgba8(kPalette[M.ids[M.offsets[geomId].x + h.primId % M.offsets[geomId].y] % 20]);
    break;
  case 8: { // NORMAL
    const f3 v = mk3(fabsf(norm.x), fabsf(norm.y), fabsf(norm.z));
    res = make_float4(0.25f + 0.5f * powf(v.x, 1.0f / 1.5f), 0.25f + 0.5f * powf(v.y, 1.0f / 1.5f),
                      0.25f + 0.5f * powf(v.z, 1.0f / 1.5f), 0.5f + 0.5f * 1.0f);
  } break;
  case 9: // BARYCENTRIC
    res = make_float4(h.coords[0], h.coords[1], 1 - h.coords[0] - h.coords[1], 1);
    break;
  case 10: // ST_ITERATIONS (primId holds the sphere-tracing steps)
    if (h.primId == 0) {
      res = make_float4(0.5f, 0.5f, 0.5f, 1.0f);
    } else if (h.primId <= 64) {
      const float q = sclamp(float(h.primId) / 64, 0.0f, 1.0f);
      res = make_float4(q * 0 + (1.0f - q) * 0, q * 0 + (1.0f - q) * 1, q * 1 + (1.0f - q) * 0, q * 1 + (1.0f - q) * 1);
    } else {
      const float q = sclamp(float(h.primId - 64) / (256 - 64), 0.0f, 1.0f);
      res = make_float4(q * 1 + (1.0f - q) * 0, q * 0 + (1.0f - q) * 0, q * 0 + (1.0f - q) * 1, q * 1 + (1.0f - q) * 1);
    }
    break;
  case 24: // MO_VOXEL_COUNT
    if (h.primId == 0) res = make_float4(0.5f, 0.5f, 0.5f, 1);
    else if (h.primId == 1) res = make_float4(0.5f, 1, 0.5f, 1);
    else if (h.primId == 2) res = make_float4(0.5f, 0.5f, 1, 1);
    else if (h.primId <= 64) {
      const float q = sclamp(float(h.primId) / 64, 0.0f, 1.0f);
      res = make_float4(q * 1 + (1 - q) * 0.5f, q * 0 + (1 - q) * 0.5f, q * 0 + (1 - q) * 1, q * 1 + (1 - q) * 1);
    } else {
      res = make_float4(1, 0, 0, 1);
    }
    break;
  case 19: { // HSV_DEPTH
    const f3 isect = rayPos + z * rayDir;
    float zt = (isect.z + 1.f) * 2.f;
    zt = zt - float(int(zt));
    if (zt < 0.f) zt = 1.f + zt;
    const float hx = zt, hy = 1.f, hz = 1.f;
    float col[4] = {hz, hz, hz, 1.f};
    const float vmin = (1.f - hy) * hz;
    const float x6 = hx * 6.f;
    const float Hi = truncf(x6);
    const float a = (hz - vmin) * (x6 - Hi);
    uint32_t H = uint32_t(Hi);
    H = H <= 5u ? H : 5u;
    col[(2u + (H >> 1)) % 3u] = vmin;
    if ((H & 1u) != 0u) col[H >> 1] = hz - a;
    else col[(1u + (H >> 1)) % 3u] = vmin + a;
    res = make_float4(col[0], col[1], col[2], 1.f);
  } break;
  case 16: { // DIFFUSE (colored materials)
    float4 col = make_float4(0, 0, 1, 1);
    if (type == LRT_TYPE_SDF_SBS_COL) {
      const f3 pc = packed_hit_colour(h);
      col = make_float4(pc.x, pc.y, pc.z, col.w);
    } else {
      col = material_colour(material());
    }
    res = make_float4(col.x, col.y, col.z, 1);
  } break;
  case 15: // TEX_COORDS
    res = make_float4(tcu, tcv, 0, 1);
    break;
  case 1:  // LAMBERT_NO_TEX
  case 13: // OUTLINE_PRIM: ResolveOutline (:1073-1121) never sets its outline flag in this mode
  case 7:  // GEOM
  case 17: // LAMBERT (colored materials)
  case 20: { // LOD
    f3 color = mk3(0, 0, 1);
    if (mode == 1 || mode == 13) color = mk3(1, 1, 1);
    else if (mode == 20) color = ld3(decode_rgba8(kLodPalette[h.primId % 20]));
    else if (mode == 7) color = ld3(decode_rgba8(kPalette[geomId % 20]));
    else if (type == LRT_TYPE_SDF_SBS_COL || type == LRT_TYPE_GRAPHICS_PRIM) color = packed_hit_colour(h);
    else color = ld3(material_colour(material()));
    const f3 fc = lambert_lights(L, norm, color, rayPos, rayDir, h.t);
    res = make_float4(fc.x, fc.y, fc.z, 1);
  } break;
  case 11: // PBR_NO_TEX (material 0, DEFAULT_MATERIAL)
  case 21: { // PBR (colored materials)
    const lrt_material& m = mode == 11 ? M.mats[0] : material();
    const f3 baseColor = ld3(material_colour(m));
    const float metallic = m.metallic, roughness = m.roughness;
    const float alpha = roughness * roughness, f0 = 0.04f, kPi = 3.14159265358979323846f; // LiteMath's M_PI, a float
    const f3 surf = rayPos + h.t * rayDir;
    const f3 eye_dir = -1.0f * rayDir;
    const float NV = dot(norm, eye_dir);
    f3 fc = mk3(0, 0, 0);
    for (uint32_t i = 0; i < L.count; i++) {
      const DevLight& l = L.light[i];
      f3 light_dir = mk3(1, 1, 1);
      if (l.type == LRT_LIGHT_DIRECT) {
        light_dir = mk3(l.space[0], l.space[1], l.space[2]);
      } else if (l.type == LRT_LIGHT_POINT) {
        light_dir = mk3(l.space[0], l.space[1], l.space[2]) - surf;
        const float len = sqrtf(dot(light_dir, light_dir));
        light_dir = mk3(light_dir.x / len, light_dir.y / len, light_dir.z / len);
      }
      f3 half = eye_dir + light_dir;
      const float hl = sqrtf(dot(half, half));
      half = mk3(half.x / hl, half.y / hl, half.z / hl);
      const float NH = dot(norm, half), NL = dot(norm, light_dir), HL = dot(half, light_dir), HV = dot(half, eye_dir);
      const float D = alpha * smax(0.0f, NH) / smax(kPi * powf(NH * NH * (alpha - 1.0f) + 1.0f, 2.0f), 0.00001f);
      float V = smax(0.0f, HL) / smax(fabsf(NL) + sqrtf(alpha + (1 - alpha) * NL * NL), 0.00001f);
      V *= smax(0.0f, HV) / smax(fabsf(NV) + sqrtf(alpha + (1 - alpha) * NV * NV), 0.00001f);
      const float spec = V * D;
      const float ip = 1.0f / kPi;
      const f3 diffuse = mk3(ip * baseColor.x, ip * baseColor.y, ip * baseColor.z);
      const float p5 = powf(1.0f - fabsf(HV), 5.0f);
      const f3 metal = spec * mk3(baseColor.x + (1.0f - baseColor.x) * p5, baseColor.y + (1.0f - baseColor.y) * p5,
                                  baseColor.z + (1.0f - baseColor.z) * p5);
      const float F = f0 + (1.0f - f0) * p5;
      const float fs = F * spec;
      const f3 diel = mk3((1.0f - F) * diffuse.x + fs, (1.0f - F) * diffuse.y + fs, (1.0f - F) * diffuse.z + fs);
      const f3 brdf = (1.0f - metallic) * diel + metallic * metal;
      fc = fc + brdf * smax(NL, 0.0f);
    }
    res = make_float4(fc.x, fc.y, fc.z, 1);
  } break;
  case 12: // PHONG_NO_TEX
  case 18: { // PHONG (colored materials); the reference's shadow ray is commented out (shade = 1)
    const float Kd = 0.25f, Ks = 0.25f, BIAS = 1e-6f;
    f3 color = mk3(0, 0, 1);
    if (mode == 12) color = mk3(1, 1, 1);
    else if (type == LRT_TYPE_SDF_SBS_COL || type == LRT_TYPE_GRAPHICS_PRIM) color = packed_hit_colour(h);
    else color = ld3(material_colour(material()));
    f3 fc = mk3(0, 0, 0);
    for (uint32_t i = 0; i < L.count; i++) {
      const DevLight& l = L.light[i];
      const f3 lc = mk3(l.color[0], l.color[1], l.color[2]);
      const f3 sp = mk3(l.space[0], l.space[1], l.space[2]);
      if (l.type == LRT_LIGHT_AMBIENT) {
        fc = fc + lc * color;
        continue;
      }
      const f3 surf = rayPos + (h.t - BIAS) * rayDir;
      f3 light_dir = mk3(1, 1, 1);
      if (l.type == LRT_LIGHT_DIRECT) {
        light_dir = sp;
        const float q = smax(0.0f, dot(norm, sp));
        fc = fc + (lc * color) * q;
      } else if (l.type == LRT_LIGHT_POINT) {
        const f3 dir = sp - surf;
        const float len = sqrtf(dot(dir, dir));
        light_dir = mk3(dir.x / len, dir.y / len, dir.z / len);
      }
      const f3 refl = -1.0f * light_dir + (2.0f * dot(norm, light_dir)) * norm;
      // Kd * max(0, n.l) + Ks * pow(max(0, n.r), 32): pow(float, int) is the
      // double overload, so the sum is formed in double and rounded once
      const double spec = double(Ks) * pow(double(smax(0.0f, dot(norm, refl))), 32.0);
      const float k = float(double(Kd * smax(0.0f, dot(norm, light_dir))) + spec);
      fc = fc + ((1.0f * lc) * k) * color;
    }
    res = make_float4(fc.x, fc.y, fc.z, 1);
  } break;
  default:
    break;
  }
  return make_float4(res.x, res.y, res.z, 1.0f);
}

// Batched multi-camera form: one persistent launch over the pixel tiles of
// all cameras.  A warp takes one tile at a time from the global counter,
// finds its camera by binary search over the tile bases, and each lane
// generates (lrt::eye_ray, the function k_eye_rays uses) and traces its
// raysPerLane pixels, so every hit equals the plain per-camera path's.
//
// RENDER: instead of hits, each pixel's RGBA8 colour (resolve_rgba8: the
// LAMBERT_NO_TEX resolve with L and the tonemap) goes to image[rayOffset + y*width + x].
template <bool RENDER>
__global__ void __launch_bounds__(kTraceThreads, 7) k_trace_cameras(DevScene S, const DevBatchCamera* __restrict__ cams,
                                                                 uint32_t ncams, uint32_t ntiles, DevBatchShape shape,
                                                                 lrt_hit* __restrict__ hits,
                                                                 unsigned long long* __restrict__ work_counter,
                                                                 uint32_t* __restrict__ err_word, DevLights L,
                                                                 uint32_t* __restrict__ image)
{
  extern __shared__ uint32_t smem_stack[];
  l2_prefetch_scene(S);
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  Ctx<false> c(S, normal_words(smem_stack, shape.stackCap));
  for (;;) {
    unsigned long long tile = 0;
    if (lane == 0) tile = atomicAdd(work_counter, 1ull);
    tile = __shfl_sync(0xFFFFFFFFu, tile, 0);
    if (tile >= ntiles) break;
    // camera of this tile: the last camera whose tileBase <= tile (uniform in the warp)
    uint32_t lo = 0, hi = ncams - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (__ldg(&cams[mid].tileBase) <= tile) lo = mid;
      else hi = mid - 1;
    }
    const DevBatchCamera& bc = cams[lo];
    const uint32_t local = uint32_t(tile) - bc.tileBase;
    const uint32_t x0 = (local % bc.tilesX) * shape.tileW, y0 = (local / bc.tilesX) * shape.tileH;
    const uint32_t W = bc.cam.width, H = bc.cam.height;
    for (uint32_t r = 0; r < shape.raysPerLane; r++) {
      const uint32_t i = lane + 32 * r;
      const uint32_t x = x0 + i % shape.tileW, y = y0 + i / shape.tileW;
      if (x >= W || y >= H) continue;
      float ray[8];
      eye_ray(bc.cam.proj_inv, bc.cam.world_view_inv, x, y, W, H, bc.cam.tnear, bc.cam.tfar, ray);
      lrt_hit h;
      trace_one(c, stack, blockDim.x, shape.stackCap, make_float4(ray[0], ray[1], ray[2], ray[3]),
                make_float4(ray[4], ray[5], ray[6], ray[7]), h);
      if (RENDER) {
        image[bc.rayOffset + uint64_t(y) * W + x] =
            resolve_rgba8(c, L, mk3(ray[0], ray[1], ray[2]), mk3(ray[4], ray[5], ray[6]), h);
      } else {
        float4* out = reinterpret_cast<float4*>(hits + bc.rayOffset + uint64_t(y) * W + x);
        out[0] = make_float4(h.t, __uint_as_float(h.primId), __uint_as_float(h.instId), __uint_as_float(h.geomId));
        out[1] = make_float4(h.coords[0], h.coords[1], h.coords[2], h.coords[3]);
      }
    }
  }
  if (c.err) atomicOr(err_word, c.err);
}

cudaError_t launch_trace_cameras(const DevScene& S, const DevBatchCamera* cams, uint32_t ncams, uint32_t ntiles,
                                 const DevBatchShape& shape, lrt_hit* hits, unsigned long long* work_counter,
                                 uint32_t* err_word, int grid, cudaStream_t stream, const DevLights* lights,
                                 uint32_t* image)
{
  const size_t smem = trace_smem_bytes(shape.stackCap);
  if (image) {
    cudaError_t e = cudaFuncSetAttribute(k_trace_cameras<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(trace_smem_bytes(kMaxStackDev + 1)));
    if (e != cudaSuccess) return e;
    k_trace_cameras<true><<<grid, kTraceThreads, smem, stream>>>(S, cams, ncams, ntiles, shape, hits, work_counter,
                                                                 err_word, *lights, image);
  } else {
    k_trace_cameras<false><<<grid, kTraceThreads, smem, stream>>>(S, cams, ncams, ntiles, shape, hits, work_counter,
                                                                  err_word, DevLights{}, nullptr);
  }
  return cudaGetLastError();
}

cudaError_t cameras_occupancy(uint32_t stack_cap, int* blocks_per_sm)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  cudaError_t e = cudaFuncSetAttribute(k_trace_cameras<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(trace_smem_bytes(kMaxStackDev + 1)));
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_trace_cameras<false>, kTraceThreads, smem);
}

// Lambert shading of a hit, MultiRenderer::ResolveCommon for
// LAMBERT_NO_TEX with one directional light of unit colour and albedo 1
// (MultiRenderer_resolve.cpp:617-666): max(0, n . L) with n decoded from the
// hit's octahedral normal (loadNormalTcFromGbuffer, :27-75); background 0.
// Triangle normals are decoded too and turned towards the viewer.
__device__ __forceinline__ float lambert(const lrt_hit& h, f3 dir, f3 L)
{
  if (h.primId == 0xFFFFFFFFu) return 0.0f;
  f3 n = decode_normal(mk2(h.coords[2], h.coords[3]));
  if ((h.geomId >> 24) == LRT_TYPE_MESH_TRIANGLE) n = ssign(dot(-1.0f * dir, n)) * n;
  return smax(0.0f, dot(n, L));
}

// MultiRenderer::Render for MULTI_RENDER_MODE_LAMBERT_NO_TEX with one sample
// per pixel and no transparency (MultiRenderer.cpp:14-60), fused into one
// launch: per pixel initEyeRay (the eye_ray of lrt_generate_eye_rays), the
// nearest hit, ResolveCommon (MultiRenderer_resolve.cpp:580-666: white albedo,
// direct / point / ambient lights, triangle normals recomputed from the
// triangle and turned towards the viewer as in loadNormalTcFromGbuffer :27-75,
// SDF normals decoded from the hit) and Tonemap (:536-542) into RGBA8.  A warp
// takes 8x4-pixel tiles from a global counter.
// MINB as for k_trace: 6 (80 registers) for one LAMBERT_NO_TEX sample of a
// scene whose geometries are all sparse-brick sets, else 7 (72 registers).
template <bool MODES, int MINB = 7>
__global__ void __launch_bounds__(kTraceThreads, MINB) k_render_rgba8(DevScene S, DevCamera cam, DevLights L,
                                                                uint32_t* __restrict__ image,
                                                                unsigned long long* __restrict__ work_counter,
                                                                uint32_t* __restrict__ err_word, uint32_t stack_cap,
                                                                const uint32_t* __restrict__ sched_rd,
                                                                uint32_t* sched_wr, DevMaterials M, DevRenderModes RM)
{
  extern __shared__ uint32_t smem_stack[];
  l2_prefetch_scene(S);
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  Ctx<false> c(S, normal_words(smem_stack, stack_cap));
  const uint32_t tilesX = (cam.width + 7) / 8, ntiles = tilesX * ((cam.height + 3) / 4);
  __shared__ WarpClock wclock[kTraceThreads / 32];
  if (lane == 0) {
    wclock[threadIdx.x >> 5].item = ~0u;
    wclock[threadIdx.x >> 5].longest = 0;
    wclock[threadIdx.x >> 5].busy = 0;
  }
  for (;;) {
    uint32_t item = 0;
    __syncwarp();
    if (lane == 0) item = sched_next(sched_rd, sched_wr, ntiles, work_counter, wclock[threadIdx.x >> 5]);
    item = __shfl_sync(0xFFFFFFFFu, item, 0);
    if (item == ~0u) break;
    const uint32_t tile = item_tile(item);
    const uint32_t x = (tile % tilesX) * 8 + (lane & 7), y = (tile / tilesX) * 4 + (lane >> 3);
    if (x < cam.width && y < cam.height && item_has_lane(item, lane)) {
      float r[8];
      eye_ray(cam.proj_inv, cam.world_view_inv, x, y, cam.width, cam.height, cam.tnear, cam.tfar, r);
      lrt_hit h;
      if (!MODES) {
        trace_one(c, stack, blockDim.x, stack_cap, make_float4(r[0], r[1], r[2], r[3]),
                  make_float4(r[4], r[5], r[6], r[7]), h);
        image[uint64_t(y) * cam.width + x] = resolve_rgba8(c, L, mk3(r[0], r[1], r[2]), mk3(r[4], r[5], r[6]), h);
      } else {
        // Render's sample loop (MultiRenderer.cpp:21-64): sample s traces the
        // ray through initEyeRay's point s of the pixel; the resolve takes the
        // sample-0 ray (ResolveCommon calls initEyeRay with sample 0) and,
        // in the transparency path, blends with the composited layers
        // (ResolveTransparency, MultiRenderer_resolve.cpp:573-577); the
        // colours are summed and the sum divided by the sample count.
        float r0[8];
        eye_ray(cam.proj_inv, cam.world_view_inv, x, y, cam.width, cam.height, cam.tnear, cam.tfar, r0,
                RM.random ? RM.randomX : RM.invSqrt * 0.5f, RM.random ? RM.randomY : RM.invSqrt * 0.5f);
        const f3 rp0 = mk3(r0[0], r0[1], r0[2]), rd0 = mk3(r0[4], r0[5], r0[6]);
        float4 acc = make_float4(0, 0, 0, 0);
        for (uint32_t smp = 0; smp < RM.samples; smp++) {
          float rs[8];
          float dx = RM.randomX, dy = RM.randomY;
          if (!RM.random) {
            dx = RM.invSqrt * float(double(smp / RM.sqrtSpp) + 0.5);
            dy = RM.invSqrt * float(double(smp % RM.sqrtSpp) + 0.5);
          }
          eye_ray(cam.proj_inv, cam.world_view_inv, x, y, cam.width, cam.height, cam.tnear, cam.tfar, rs, dx, dy);
          f3 tc = mk3(0, 0, 0);
          float alpha = 1.0f;
          if (RM.transparency)
            anyhit_loop(c, stack, stack_cap, M, rs, h, tc, alpha);
          else
            trace_one(c, stack, blockDim.x, stack_cap, make_float4(rs[0], rs[1], rs[2], rs[3]),
                      make_float4(rs[4], rs[5], rs[6], rs[7]), h);
          float4 col = resolve_mode_colour(c, L, M, RM.mode, rp0, rd0, h);
          if (RM.transparency) col = make_float4(tc.x + alpha * col.x, tc.y + alpha * col.y, tc.z + alpha * col.z, col.w);
          acc = smp == 0 ? col : make_float4(acc.x + col.x, acc.y + col.y, acc.z + col.z, acc.w + col.w);
        }
        const float ns = float(RM.samples);
        image[uint64_t(y) * cam.width + x] = tonemap_rgba8(acc.x / ns, acc.y / ns, acc.z / ns, acc.w / ns);
      }
    }
  }
  if (c.err) atomicOr(err_word, c.err);
}

// OUTLINE_BORDER (MultiRenderer.cpp:55-58: FillGbuffer, then ResolveOutline,
// MultiRenderer_resolve.cpp:1073-1128), the G-buffer pass of sample smp: per
// pixel the nearest hit of the sample's ray — its t and whether it missed
// (tm) — and the pixel's colour before the outline test (col): white Lambert
// of the hit under the lights, shaded with the sample-0 ray as ResolveOutline
// does (the OUTLINE_PRIM colour), or the background for a miss.  The colour
// is resolved here, with the trace's context, because a triangle's normal
// needs the triangle record the traversal found.
__global__ void __launch_bounds__(kTraceThreads, 7) k_outline_fill(DevScene S, DevCamera cam, DevLights L,
                                                                DevMaterials M, DevRenderModes RM, uint32_t smp,
                                                                float2* __restrict__ tm, float4* __restrict__ col,
                                                                unsigned long long* __restrict__ work_counter,
                                                                uint32_t* __restrict__ err_word, uint32_t stack_cap,
                                                                const uint32_t* __restrict__ sched_rd,
                                                                uint32_t* sched_wr)
{
  extern __shared__ uint32_t smem_stack[];
  l2_prefetch_scene(S);
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  Ctx<false> c(S, normal_words(smem_stack, stack_cap));
  const uint32_t tilesX = (cam.width + 7) / 8, ntiles = tilesX * ((cam.height + 3) / 4);
  __shared__ WarpClock wclock[kTraceThreads / 32];
  if (lane == 0) {
    wclock[threadIdx.x >> 5].item = ~0u;
    wclock[threadIdx.x >> 5].longest = 0;
    wclock[threadIdx.x >> 5].busy = 0;
  }
  for (;;) {
    uint32_t item = 0;
    __syncwarp();
    if (lane == 0) item = sched_next(sched_rd, sched_wr, ntiles, work_counter, wclock[threadIdx.x >> 5]);
    item = __shfl_sync(0xFFFFFFFFu, item, 0);
    if (item == ~0u) break;
    const uint32_t tile = item_tile(item);
    const uint32_t x = (tile % tilesX) * 8 + (lane & 7), y = (tile / tilesX) * 4 + (lane >> 3);
    if (x < cam.width && y < cam.height && item_has_lane(item, lane)) {
      float r0[8], rs[8];
      eye_ray(cam.proj_inv, cam.world_view_inv, x, y, cam.width, cam.height, cam.tnear, cam.tfar, r0,
              RM.random ? RM.randomX : RM.invSqrt * 0.5f, RM.random ? RM.randomY : RM.invSqrt * 0.5f);
      float dx = RM.randomX, dy = RM.randomY;
      if (!RM.random) {
        dx = RM.invSqrt * float(double(smp / RM.sqrtSpp) + 0.5);
        dy = RM.invSqrt * float(double(smp % RM.sqrtSpp) + 0.5);
      }
      eye_ray(cam.proj_inv, cam.world_view_inv, x, y, cam.width, cam.height, cam.tnear, cam.tfar, rs, dx, dy);
      lrt_hit h;
      trace_one(c, stack, blockDim.x, stack_cap, make_float4(rs[0], rs[1], rs[2], rs[3]),
                make_float4(rs[4], rs[5], rs[6], rs[7]), h);
      const uint64_t p = uint64_t(y) * cam.width + x;
      tm[p] = make_float2(h.t, h.primId == 0xFFFFFFFFu ? 1.0f : 0.0f);
      col[p] = resolve_mode_colour(c, L, M, LRT_RENDER_MODE_OUTLINE_PRIM, mk3(r0[0], r0[1], r0[2]),
                                   mk3(r0[4], r0[5], r0[6]), h);
    }
  }
  if (c.err) atomicOr(err_word, c.err);
}

// ResolveOutline's test (MultiRenderer_resolve.cpp:1112-1127) and the sum over
// samples: a hit pixel whose t differs from the t of one of its four
// neighbours (the pixel itself at the image's edges) by more than
// 10 t / width takes (0.2, 0.2, 0.2, 1); misses keep the background.  The
// last sample's pass divides the sum by the sample count and tonemaps.
__global__ void __launch_bounds__(256) k_outline_resolve(const float2* __restrict__ tm, const float4* __restrict__ col,
                                                         uint32_t w, uint32_t h, uint32_t smp, uint32_t samples,
                                                         float4* __restrict__ acc, uint32_t* __restrict__ image)
{
  const uint64_t n = uint64_t(w) * h;
  for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < n; p += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t x = uint32_t(p % w), y = uint32_t(p / w);
    const float2 me = tm[p];
    float4 c = col[p];
    if (me.y == 0.0f) {
      const float t = me.x;
      const float tol = 10.0f * t / float(w);
      const float tl = tm[x == 0 ? p : p - 1].x, tu = tm[y == 0 ? p : p - w].x;
      const float tr = tm[x == w - 1 ? p : p + 1].x, td = tm[y == h - 1 ? p : p + w].x;
      if (fabsf(tl - t) > tol || fabsf(tu - t) > tol || fabsf(tr - t) > tol || fabsf(td - t) > tol)
        c = make_float4(0.2f, 0.2f, 0.2f, 1.0f);
    }
    if (smp) {
      const float4 a = acc[p];
      c = make_float4(a.x + c.x, a.y + c.y, a.z + c.z, a.w + c.w);
    }
    if (smp + 1 < samples) {
      acc[p] = c;
    } else {
      const float ns = float(samples);
      image[p] = tonemap_rgba8(c.x / ns, c.y / ns, c.z / ns, c.w / ns);
    }
  }
}

// kernel1D_FillGbufferWithTransparency (MultiRenderer.cpp:204-221) for one
// sample: anyhit_loop per pixel of the camera (8x4-pixel tiles per warp).
__global__ void __launch_bounds__(kTraceThreads, 7) k_fill_gbuffer_transparency(
    DevScene S, DevCamera cam, DevMaterials M, float4* __restrict__ transparency, lrt_hit* __restrict__ gbuffer,
    unsigned long long* __restrict__ work_counter, uint32_t* __restrict__ err_word, uint32_t stack_cap,
    const uint32_t* __restrict__ sched_rd, uint32_t* sched_wr)
{
  extern __shared__ uint32_t smem_stack[];
  l2_prefetch_scene(S);
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  Ctx<false> c(S, normal_words(smem_stack, stack_cap));
  const uint32_t tilesX = (cam.width + 7) / 8, ntiles = tilesX * ((cam.height + 3) / 4);
  __shared__ WarpClock wclock[kTraceThreads / 32];
  if (lane == 0) {
    wclock[threadIdx.x >> 5].item = ~0u;
    wclock[threadIdx.x >> 5].longest = 0;
    wclock[threadIdx.x >> 5].busy = 0;
  }
  for (;;) {
    uint32_t item = 0;
    __syncwarp();
    if (lane == 0) item = sched_next(sched_rd, sched_wr, ntiles, work_counter, wclock[threadIdx.x >> 5]);
    item = __shfl_sync(0xFFFFFFFFu, item, 0);
    if (item == ~0u) break;
    const uint32_t tile = item_tile(item);
    const uint32_t x = (tile % tilesX) * 8 + (lane & 7), y = (tile / tilesX) * 4 + (lane >> 3);
    if (x < cam.width && y < cam.height && item_has_lane(item, lane)) {
      float r[8];
      eye_ray(cam.proj_inv, cam.world_view_inv, x, y, cam.width, cam.height, cam.tnear, cam.tfar, r);
      lrt_hit h;
      f3 tc;
      float alpha;
      anyhit_loop(c, stack, stack_cap, M, r, h, tc, alpha);
      const uint64_t i = uint64_t(y) * cam.width + x;
      transparency[i] = make_float4(tc.x, tc.y, tc.z, alpha);
      float4* out = reinterpret_cast<float4*>(gbuffer + i);
      out[0] = make_float4(h.t, __uint_as_float(h.primId), __uint_as_float(h.instId), __uint_as_float(h.geomId));
      out[1] = make_float4(h.coords[0], h.coords[1], h.coords[2], h.coords[3]);
    }
  }
  if (c.err) atomicOr(err_word, c.err);
}

// The next ray of this lane for the Lambert passes; false (warp-uniform) when
// the launch's work is done.  IMG: the rays are an img_w x img_h image in
// row-major pixel order and the warp takes its next 8x4-pixel tile from the
// stream's tile schedule (as k_trace does); otherwise the next 32 rays of n.
// `valid` is false for the lanes of a tile past the image's edge or past n.
template <bool IMG>
__device__ __forceinline__ bool next_ray(uint64_t n, uint32_t img_w, uint32_t img_h, unsigned long long* counter,
                                         const uint32_t* sched_rd, uint32_t* sched_wr, WarpClock* wc, uint64_t& i,
                                         bool& valid)
{
  const uint32_t lane = threadIdx.x & 31;
  if (IMG) {
    const uint32_t tilesX = (img_w + kImgTileW - 1) / kImgTileW;
    __syncwarp();
    uint32_t item = 0;
    if (lane == 0) item = sched_next(sched_rd, sched_wr, tilesX * ((img_h + kImgTileH - 1) / kImgTileH), counter, *wc);
    item = __shfl_sync(0xFFFFFFFFu, item, 0);
    if (item == ~0u) return false;
    const uint32_t tile = item_tile(item);
    const uint32_t x = (tile % tilesX) * kImgTileW + lane % kImgTileW;
    const uint32_t y = (tile / tilesX) * kImgTileH + lane / kImgTileW;
    valid = x < img_w && y < img_h && item_has_lane(item, lane);
    i = uint64_t(y) * img_w + x;
    valid = valid && i < n; // ray-order rays traced as an 8-wide image have a ragged last row
    return true;
  }
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(counter, 32ull);
  base = __shfl_sync(0xFFFFFFFFu, base, 0);
  if (base >= n) return false;
  i = base + lane;
  valid = i < n;
  return true;
}

// Forward render: image[i] = Lambert shade of ray i's nearest hit.
template <bool IMG>
__global__ void __launch_bounds__(kTraceThreads, 7) k_render_lambert(DevScene S, const float4* __restrict__ rays,
                                                                  uint64_t n, float3 light, float* __restrict__ image,
                                                                  unsigned long long* __restrict__ work_counter,
                                                                  uint32_t* __restrict__ err_word, uint32_t stack_cap,
                                                                  uint32_t img_w, uint32_t img_h,
                                                                  const uint32_t* __restrict__ sched_rd,
                                                                  uint32_t* sched_wr)
{
  extern __shared__ uint32_t smem_stack[];
  l2_prefetch_scene(S);
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  __shared__ WarpClock wclock[IMG ? kTraceThreads / 32 : 1];
  WarpClock* wc = wclock + (IMG ? threadIdx.x >> 5 : 0);
  if (IMG && lane == 0) {
    wc->item = ~0u;
    wc->longest = 0;
    wc->busy = 0;
  }
  Ctx<false> c(S, normal_words(smem_stack, stack_cap));
  const f3 L = mk3(light.x, light.y, light.z);
  uint64_t i = 0;
  bool valid = false;
  while (next_ray<IMG>(n, img_w, img_h, work_counter, sched_rd, sched_wr, wc, i, valid)) {
    if (valid) {
      const float4 pn = __ldg(rays + 2 * i), df = __ldg(rays + 2 * i + 1);
      lrt_hit h;
      trace_one(c, stack, blockDim.x, stack_cap, pn, df, h);
      image[i] = lambert(h, mk3(df.x, df.y, df.z), L);
    }
  }
  if (c.err) atomicOr(err_word, c.err);
}

// Adjoint of the render with respect to the SBS float values.  The march is
// recomputed (same traversal, recording the hit voxel), then at the hit
// point p (voxel units) of the trilinear field f(p; theta):
//   g = grad_p f,  n = M g / |M g|  (M = transformInvTransposed),
//   dt/dtheta_i = -w_i(p) / (g . dir)            (implicit differentiation),
//   dI/dtheta_i = [n.L > 0] * ( u . grad w_i(p) + (u^T H dir) dt/dtheta_i ),
//   u = M^T (1 - n n^T) L / |M g|,  H = Hessian of f at p (mixed terms only),
// and dLoss/dI * dI/dtheta_i is added to grad[idx_i] for the 8 corners.
// Rays whose dLoss/dI is 0 are skipped.  Hits off indexed SBS bricks
// contribute nothing.
template <bool IMG>
__global__ void __launch_bounds__(kTraceThreads, 7) k_adjoint_lambert(DevScene S, const float4* __restrict__ rays,
                                                                   uint64_t n, float3 light,
                                                                   const float* __restrict__ dimage,
                                                                   float* __restrict__ grad,
                                                                   unsigned long long* __restrict__ work_counter,
                                                                   uint32_t* __restrict__ err_word, uint32_t stack_cap,
                                                                   uint32_t img_w, uint32_t img_h,
                                                                   const uint32_t* __restrict__ sched_rd,
                                                                   uint32_t* sched_wr)
{
  extern __shared__ uint32_t smem_stack[];
  l2_prefetch_scene(S);
  uint32_t* stack = smem_stack + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  __shared__ WarpClock wclock[IMG ? kTraceThreads / 32 : 1];
  WarpClock* wc = wclock + (IMG ? threadIdx.x >> 5 : 0);
  if (IMG && lane == 0) {
    wc->item = ~0u;
    wc->longest = 0;
    wc->busy = 0;
  }
  const f3 L = mk3(light.x, light.y, light.z);
  uint32_t err = 0;
  uint64_t i = 0;
  bool valid = false;
  while (next_ray<IMG>(n, img_w, img_h, work_counter, sched_rd, sched_wr, wc, i, valid)) {
    if (!valid) continue;
    const float dLdI = __ldg(dimage + i);
    if (dLdI == 0.0f) continue;
    Ctx<false, true> c(S, normal_words(smem_stack, stack_cap));
    const float4 pn = __ldg(rays + 2 * i), df = __ldg(rays + 2 * i + 1);
    lrt_hit h;
    trace_one(c, stack, blockDim.x, stack_cap, pn, df, h);
    err |= c.err;
    if (h.primId == 0xFFFFFFFFu || !c.rec.sbs || c.rec.t != h.t) continue;
    if (lambert(h, mk3(df.x, df.y, df.z), L) <= 0.0f) continue; // max(0, .) is flat there
    const HitRecord& r = c.rec;
    const float* M = S.instances[h.instId].transformInvTransposed;
    const f3 p = r.p;
    // trilinear gradient and mixed second derivatives at p
    f3 g = mk3(0, 0, 0);
    float hxy = 0, hxz = 0, hyz = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float sx = (k & 4) ? 1.0f : -1.0f, sy = (k & 2) ? 1.0f : -1.0f, sz = (k & 1) ? 1.0f : -1.0f;
      const float wx = (k & 4) ? p.x : 1.0f - p.x, wy = (k & 2) ? p.y : 1.0f - p.y, wz = (k & 1) ? p.z : 1.0f - p.z;
      const float v = r.values[k];
      g = g + v * mk3(sx * wy * wz, wx * sy * wz, wx * wy * sz);
      hxy += v * sx * sy * wz;
      hxz += v * sx * wy * sz;
      hyz += v * wx * sy * sz;
    }
    const f3 m = matmul4(M, g, 0.0f);
    const float inv_len = 1.0f / sqrtf(dot(m, m));
    const f3 nn = inv_len * m;
    const f3 q = inv_len * (L - dot(nn, L) * nn); // (1 - n n^T) L / |M g|
    // u = M^T q (M column-major: M^T q has components dot(column_k, q))
    const f3 u = mk3(M[0] * q.x + M[1] * q.y + M[2] * q.z, M[4] * q.x + M[5] * q.y + M[6] * q.z,
                     M[8] * q.x + M[9] * q.y + M[10] * q.z);
    const f3 dir = r.dir;
    const f3 Hd = mk3(hxy * dir.y + hxz * dir.z, hxy * dir.x + hyz * dir.z, hxz * dir.x + hyz * dir.y);
    const float gd = dot(g, dir);
    if (gd == 0.0f && !r.early) continue;
    const float uHd = r.early ? 0.0f : dot(u, Hd); // early hits: the hit point is fixed
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const float sx = (k & 4) ? 1.0f : -1.0f, sy = (k & 2) ? 1.0f : -1.0f, sz = (k & 1) ? 1.0f : -1.0f;
      const float wx = (k & 4) ? p.x : 1.0f - p.x, wy = (k & 2) ? p.y : 1.0f - p.y, wz = (k & 1) ? p.z : 1.0f - p.z;
      const float w = wx * wy * wz;
      const f3 dw = mk3(sx * wy * wz, wx * sy * wz, wx * wy * sz);
      const float dI = r.early ? dot(u, dw) : dot(u, dw) - uHd * w / gd;
      atomicAdd(grad + r.idx[k], dLdI * dI);
    }
  }
  if (err) atomicOr(err_word, err);
}

cudaError_t launch_render_rgba8(const DevScene& S, const DevCamera& cam, const DevLights& lights, uint32_t* image,
                                unsigned long long* work_counter, uint32_t* err_word, uint32_t stack_cap, int grid,
                                cudaStream_t stream, const uint32_t* sched_rd, uint32_t* sched_wr,
                                const DevMaterials* materials, const DevRenderModes* rm, bool bricks_only)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  // one sample of LAMBERT_NO_TEX keeps its own instantiation (the benchmarked
  // render; bounded to 80 registers for brick-only scenes); the other modes,
  // several samples and transparency share the general one
  const bool modes = rm && (rm->mode != LRT_RENDER_MODE_LAMBERT_NO_TEX || rm->samples != 1 || rm->transparency);
  auto kernel = modes ? k_render_rgba8<true> : bricks_only ? k_render_rgba8<false, 6> : k_render_rgba8<false>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(trace_smem_bytes(kMaxStackDev + 1)));
  if (e != cudaSuccess) return e;
  DevRenderModes one{};
  one.mode = LRT_RENDER_MODE_LAMBERT_NO_TEX;
  one.samples = 1;
  kernel<<<grid, kTraceThreads, smem, stream>>>(S, cam, lights, image, work_counter, err_word, stack_cap, sched_rd,
                                                sched_wr, materials ? *materials : DevMaterials{}, rm ? *rm : one);
  return cudaGetLastError();
}

cudaError_t launch_outline_fill(const DevScene& S, const DevCamera& cam, const DevLights& lights,
                               const DevMaterials& M, const DevRenderModes& RM, uint32_t smp, float2* tm, float4* col,
                               unsigned long long* work_counter, uint32_t* err_word, uint32_t stack_cap, int grid,
                               cudaStream_t stream, const uint32_t* sched_rd, uint32_t* sched_wr)
{
  cudaError_t e = cudaFuncSetAttribute(k_outline_fill, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(trace_smem_bytes(kMaxStackDev + 1)));
  if (e != cudaSuccess) return e;
  k_outline_fill<<<grid, kTraceThreads, trace_smem_bytes(stack_cap), stream>>>(
      S, cam, lights, M, RM, smp, tm, col, work_counter, err_word, stack_cap, sched_rd, sched_wr);
  return cudaGetLastError();
}

cudaError_t launch_outline_resolve(const float2* tm, const float4* col, uint32_t w, uint32_t h, uint32_t smp,
                                   uint32_t samples, float4* acc, uint32_t* image, cudaStream_t stream)
{
  const uint64_t n = uint64_t(w) * h;
  const int grid = int(std::min<uint64_t>((n + 255) / 256, 148ull * 16));
  k_outline_resolve<<<grid, 256, 0, stream>>>(tm, col, w, h, smp, samples, acc, image);
  return cudaGetLastError();
}

cudaError_t launch_fill_gbuffer_transparency(const DevScene& S, const DevCamera& cam, const DevMaterials& M,
                                             float4* transparency, lrt_hit* gbuffer, unsigned long long* work_counter,
                                             uint32_t* err_word, uint32_t stack_cap, int grid, cudaStream_t stream,
                                             const uint32_t* sched_rd, uint32_t* sched_wr)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  cudaError_t e = cudaFuncSetAttribute(k_fill_gbuffer_transparency, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(trace_smem_bytes(kMaxStackDev + 1)));
  if (e != cudaSuccess) return e;
  k_fill_gbuffer_transparency<<<grid, kTraceThreads, smem, stream>>>(S, cam, M, transparency, gbuffer, work_counter,
                                                                     err_word, stack_cap, sched_rd, sched_wr);
  return cudaGetLastError();
}

// img_w > 0: the n = img_w * img_h rays are an image (row-major pixels)
// traced in 8x4-pixel tiles in the order of the tile schedule (sched_rd,
// sched_wr; nullptr for natural order).
cudaError_t launch_render_lambert(const DevScene& S, const float4* rays, uint64_t n, float3 light, float* image,
                                  unsigned long long* work_counter, uint32_t* err_word, uint32_t stack_cap, int grid,
                                  cudaStream_t stream, uint32_t img_w, uint32_t img_h, const uint32_t* sched_rd,
                                  uint32_t* sched_wr)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  auto kernel = img_w ? k_render_lambert<true> : k_render_lambert<false>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(trace_smem_bytes(kMaxStackDev + 1)));
  if (e != cudaSuccess) return e;
  kernel<<<grid, kTraceThreads, smem, stream>>>(S, rays, n, light, image, work_counter, err_word, stack_cap, img_w,
                                                img_h, sched_rd, sched_wr);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_lambert(const DevScene& S, const float4* rays, uint64_t n, float3 light,
                                   const float* dimage, float* grad, unsigned long long* work_counter,
                                   uint32_t* err_word, uint32_t stack_cap, int grid, cudaStream_t stream,
                                   uint32_t img_w, uint32_t img_h, const uint32_t* sched_rd, uint32_t* sched_wr)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  auto kernel = img_w ? k_adjoint_lambert<true> : k_adjoint_lambert<false>;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(trace_smem_bytes(kMaxStackDev + 1)));
  if (e != cudaSuccess) return e;
  kernel<<<grid, kTraceThreads, smem, stream>>>(S, rays, n, light, dimage, grad, work_counter, err_word, stack_cap,
                                                img_w, img_h, sched_rd, sched_wr);
  return cudaGetLastError();
}

// Eye rays of one camera (MultiRenderer::initEyeRay), row-major pixels.
__global__ void k_eye_rays(DevCamera cam, float4* __restrict__ rays)
{
  const uint64_t n = uint64_t(cam.width) * cam.height;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    float r[8];
    eye_ray(cam.proj_inv, cam.world_view_inv, uint32_t(i % cam.width), uint32_t(i / cam.width), cam.width,
            cam.height, cam.tnear, cam.tfar, r);
    rays[2 * i] = make_float4(r[0], r[1], r[2], r[3]);
    rays[2 * i + 1] = make_float4(r[4], r[5], r[6], r[7]);
  }
}

// Host-side launchers (one copy per namespace; declared in trace_api.h).
cudaError_t launch_trace(const DevScene& S, const float4* rays, lrt_hit* hits, uint64_t n,
                                unsigned long long* work_counter, unsigned long long* counters, uint32_t* err_word,
                                uint32_t stack_cap, int grid, cudaStream_t stream, bool count, uint32_t img_w,
                                uint32_t img_h, const uint32_t* sched_rd, uint32_t* sched_wr, uint32_t group,
                                bool bricks_only)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  // the ANALYTIC / NEWTON / IT node solvers live in their own instantiation,
  // so that the sphere-tracing kernel keeps its registers
  const uint32_t solver = (S.flags >> kFlagSolverShift) & 7u;
  const bool solvers = solver != kSolverST && solver != kSolverBBox;
  // image order (IMG) is its own instantiation, so that the tile schedule
  // costs the row-order kernel nothing
  auto go = [&](auto kernel) {
    kernel<<<grid, kTraceThreads, smem, stream>>>(S, rays, hits, n, work_counter, counters, err_word, stack_cap, img_w,
                                                  img_h, sched_rd, sched_wr, group);
  };
  if (img_w) {
    if (count && solvers) go(k_trace<true, true, true>);
    else if (count) go(k_trace<true, false, true>);
    else if (solvers) go(k_trace<false, true, true>);
    else if (bricks_only) go(k_trace<false, false, true, 6>);
    else go(k_trace<false, false, true>);
  } else {
    if (count && solvers) go(k_trace<true, true, false>);
    else if (count) go(k_trace<true, false, false>);
    else if (solvers) go(k_trace<false, true, false>);
    else if (group < 32) go(k_trace<false, false, false, 6>); // latency-bound: fewer spills per step
    else go(k_trace<false, false, false>);
  }
  return cudaGetLastError();
}

cudaError_t set_trace_smem(uint32_t stack_cap)
{
  const int smem = int(trace_smem_bytes(stack_cap));
  cudaError_t e = cudaSuccess;
  auto set = [&](auto kernel) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  };
  set(k_trace<true, false, false>);
  set(k_trace<true, true, false>);
  set(k_trace<false, true, false>);
  set(k_trace<false, false, false>);
  set(k_trace<true, false, true>);
  set(k_trace<true, true, true>);
  set(k_trace<false, true, true>);
  set(k_trace<false, false, true>);
  set(k_trace<false, false, true, 6>);
  set(k_trace<false, false, false, 6>);
  return e;
}

cudaError_t trace_occupancy(uint32_t stack_cap, int* blocks_per_sm, bool bricks_only)
{
  const size_t smem = trace_smem_bytes(stack_cap);
  // (k_render_rgba8<false, 6> has the same bound and shared memory)
  if (bricks_only)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_trace<false, false, true, 6>,
                                                         kTraceThreads, smem);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k_trace<false, false, false>, kTraceThreads,
                                                       smem);
}

cudaError_t launch_eye_rays(const DevCamera& cam, float4* rays, cudaStream_t stream)
{
  const uint64_t n = uint64_t(cam.width) * cam.height;
  const int grid = int(std::min<uint64_t>((n + 255) / 256, 148ull * 16));
  k_eye_rays<<<grid, 256, 0, stream>>>(cam, rays);
  return cudaGetLastError();
}

} // namespace LRT_NS

// wavefront.cu — second-wavefront rays: one cosine-weighted diffuse bounce
// per primary hit (lrt_generate_bounce_rays).
//
// The bounce direction follows MapSampleToCosineDistribution with power 1
// (utils/raytracing/render_common.h:75-113) around the hit's decoded normal
// turned towards the incoming ray; the two uniforms come from a PCG hash of
// (ray index, seed).  Rays whose primary ray missed get a NaN origin: every
// box test of the traversal fails on NaN, so they miss after two TLAS node
// tests, and a caller can drop them (origin x != x) before tracing.
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "device_scene.h"
#include "lrt_math.h"

namespace lrt {
namespace {

// PCG-RXS-M-XS 32-bit output of a 64-bit LCG step (O'Neill, "PCG: A Family
// of Simple Fast Space-Efficient Statistically Good Algorithms for Random
// Number Generation", 2014).
__device__ __forceinline__ uint32_t pcg_hash(uint64_t& state)
{
  state = state * 6364136223846793005ull + 1442695040888963407ull;
  const uint32_t x = uint32_t(((state >> ((state >> 59u) + 5u)) ^ state) * 12605985483714917081ull >> 32);
  return x;
}

__device__ __forceinline__ float uniform01(uint64_t& state) { return float(pcg_hash(state) >> 8) * (1.0f / 16777216.0f); }

// CoordinateSystem, render_common.h:57-73
__device__ void coordinate_system(f3 v1, f3* v2, f3* v3)
{
  if (fabsf(v1.x) > fabsf(v1.y)) {
    const float invLen = 1.0f / sqrtf(v1.x * v1.x + v1.z * v1.z);
    *v2 = mk3(-1.0f * v1.z * invLen, 0.0f, v1.x * invLen);
  } else {
    const float invLen = 1.0f / sqrtf(v1.y * v1.y + v1.z * v1.z);
    *v2 = mk3(0.0f, v1.z * invLen, -1.0f * v1.y * invLen);
  }
  *v3 = cross(v1, *v2);
}

// MapSampleToCosineDistribution(r1, r2, direction = n, hit_norm = n, power = 1)
__device__ f3 cosine_sample(float r1, float r2, f3 n)
{
  const float two_pi = 6.283185307179586f;
  const float sin_phi = sinf(two_pi * r1), cos_phi = cosf(two_pi * r1);
  const float cos_theta = sqrtf(1.0f - r2); // pow(1 - r2, 1 / (power + 1)) for power 1
  const float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
  const f3 dev = mk3(sin_theta * cos_phi, sin_theta * sin_phi, cos_theta);
  f3 nx, nz;
  coordinate_system(n, &nx, &nz);
  const f3 ny = nz; // the reference swaps ny and nz after CoordinateSystem
  nz = n;
  f3 res = nx * dev.x + ny * dev.y + nz * dev.z;
  if (dot(res, n) < 0.0f) res = (-1.0f * nx) * dev.x + ny * dev.y - nz * dev.z;
  return res;
}

// The bounce ray of traced ray i (which hit): origin at the hit point,
// cosine-weighted direction around the normal turned towards the ray.
__device__ __forceinline__ void bounce_ray(const float4 pn, const float4 df, const float4 h0, const float4 h1,
                                           uint64_t i, uint64_t seed, float tnear, float tfar, float4* out)
{
  const f3 dir = mk3(df.x, df.y, df.z);
  const f3 pos = mk3(pn.x, pn.y, pn.z) + h0.x * dir;
  f3 nrm = decode_normal(mk2(h1.z, h1.w));
  if (dot(nrm, dir) > 0.0f) nrm = -1.0f * nrm; // face the incoming ray
  uint64_t state = (i + 1) * 0x9E3779B97F4A7C15ull ^ seed;
  pcg_hash(state);
  const float r1 = uniform01(state), r2 = uniform01(state);
  const f3 b = normalize(cosine_sample(r1, r2, nrm));
  out[0] = make_float4(pos.x, pos.y, pos.z, tnear);
  out[1] = make_float4(b.x, b.y, b.z, tfar);
}

__global__ void k_bounce(const float4* __restrict__ rays, const lrt_hit* __restrict__ hits, uint64_t n, uint64_t seed,
                         float tnear, float tfar, float4* __restrict__ out)
{
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const float4 h0 = reinterpret_cast<const float4*>(hits + i)[0];
    if (__float_as_uint(h0.y) == 0xFFFFFFFFu) {
      const float qnan = __int_as_float(0x7fc00000);
      out[2 * i] = make_float4(qnan, qnan, qnan, tnear);
      out[2 * i + 1] = make_float4(0.0f, 0.0f, 1.0f, tfar);
      continue;
    }
    const float4 h1 = reinterpret_cast<const float4*>(hits + i)[1];
    bounce_ray(rays[2 * i], rays[2 * i + 1], h0, h1, i, seed, tnear, tfar, out + 2 * i);
  }
}

// Stream compaction of the hits in three passes over tiles of kTile rays
// (kCompactThreads threads x kCompactItems rays, ray k*kCompactThreads + tid
// of the tile for item k): count the hits of each tile, scan the tile
// counts, then write each hit's bounce ray at its rank, so the output keeps
// the order of the traced rays.
constexpr int kCompactThreads = 256, kCompactItems = 8, kTile = kCompactThreads * kCompactItems;

__device__ __forceinline__ bool is_hit(const lrt_hit* hits, uint64_t i, uint64_t n)
{
  return i < n && __ldg(&hits[i].primId) != 0xFFFFFFFFu;
}

__global__ void __launch_bounds__(kCompactThreads) k_count_hits(const lrt_hit* __restrict__ hits, uint64_t n,
                                                                uint32_t* __restrict__ tile_count)
{
  __shared__ uint32_t warp_sum[kCompactThreads / 32];
  const uint64_t base = uint64_t(blockIdx.x) * kTile;
  uint32_t c = 0;
#pragma unroll
  for (int k = 0; k < kCompactItems; k++) c += is_hit(hits, base + k * kCompactThreads + threadIdx.x, n);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int w = 0; w < kCompactThreads / 32; w++) t += warp_sum[w];
    tile_count[blockIdx.x] = t;
  }
}

// Exclusive scan of the tile counts (one block); count_out = the total.
__global__ void __launch_bounds__(1024) k_scan_tiles(uint32_t* __restrict__ tile, uint32_t ntiles,
                                                     unsigned long long* __restrict__ count_out)
{
  __shared__ uint32_t warp_sum[32];
  __shared__ unsigned long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (uint32_t start = 0; start < ntiles; start += 1024) {
    const uint32_t t = start + threadIdx.x;
    const uint32_t v = t < ntiles ? tile[t] : 0;
    uint32_t x = v; // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
      if ((threadIdx.x & 31) >= uint32_t(o)) x += y;
    }
    if ((threadIdx.x & 31) == 31) warp_sum[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x < 32) {
      uint32_t w = warp_sum[threadIdx.x];
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
        if (threadIdx.x >= uint32_t(o)) w += y;
      }
      warp_sum[threadIdx.x] = w; // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = (threadIdx.x >= 32 ? warp_sum[(threadIdx.x >> 5) - 1] : 0) + (x - v);
    if (t < ntiles) tile[t] = uint32_t(carry) + before;
    __syncthreads();
    if (threadIdx.x == 0) carry += warp_sum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) *count_out = carry;
}

__global__ void __launch_bounds__(kCompactThreads)
    k_bounce_compact(const float4* __restrict__ rays, const lrt_hit* __restrict__ hits, uint64_t n, uint64_t seed,
                     float tnear, float tfar, const uint32_t* __restrict__ tile_offset, float4* __restrict__ out,
                     uint32_t* __restrict__ index)
{
  __shared__ uint32_t warp_sum[kCompactThreads / 32];
  const uint64_t base = uint64_t(blockIdx.x) * kTile;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t rank = tile_offset[blockIdx.x];
#pragma unroll 1
  for (int k = 0; k < kCompactItems; k++) {
    const uint64_t i = base + k * kCompactThreads + threadIdx.x;
    const bool h = is_hit(hits, i, n);
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, h);
    if (lane == 0) warp_sum[warp] = __popc(m);
    __syncthreads();
    uint32_t before = 0, total = 0;
    for (int w = 0; w < kCompactThreads / 32; w++) {
      const uint32_t c = warp_sum[w];
      before += (w < int(warp)) ? c : 0;
      total += c;
    }
    if (h) {
      const uint32_t pos = rank + before + __popc(m & ((1u << lane) - 1u));
      const float4 h0 = reinterpret_cast<const float4*>(hits + i)[0];
      const float4 h1 = reinterpret_cast<const float4*>(hits + i)[1];
      bounce_ray(rays[2 * i], rays[2 * i + 1], h0, h1, i, seed, tnear, tfar, out + 2 * uint64_t(pos));
      index[pos] = uint32_t(i);
    }
    rank += total;
    __syncthreads();
  }
}

// Coherence key of a hit's bounce ray (lrt_generate_bounce_rays_sorted): the
// cell of the direction in a 4x4x4 grid over [-1, 1]^3 (bits 18..23) above
// the Morton code of the origin on a 64^3 grid over the scene box (bits
// 0..17, x highest of each triple), at most kMissKey - 1; misses get
// kMissKey and sort last.  24 bits: three passes of the radix sort.  Every
// rounding is an explicit IEEE round-to-nearest operation (no contraction),
// so a host restatement in float32 computes the same key.
constexpr uint32_t kMissKey = 0xFFFFFFu;
constexpr int kKeyBits = 24;

__device__ __forceinline__ uint32_t spread3_6(uint32_t x)
{
  x &= 0x3Fu;
  x = (x | (x << 8)) & 0x0000F00Fu;
  x = (x | (x << 4)) & 0x000C30C3u;
  x = (x | (x << 2)) & 0x00249249u;
  return x;
}

__device__ __forceinline__ uint32_t dir_cell(float d)
{
  const float g = __fmul_rn(__fadd_rn(d, 1.0f), 2.0f);
  return !(g > 0.0f) ? 0u : g >= 3.0f ? 3u : uint32_t(g);
}

__device__ __forceinline__ uint32_t box_cell(float o, float lo, float scale)
{
  const float f = __fmul_rn(__fsub_rn(o, lo), scale);
  return !(f > 0.0f) ? 0u : f >= 63.0f ? 63u : uint32_t(f);
}

__device__ __forceinline__ uint32_t coherence_key(const float4* b, float3 lo, float3 scale)
{
  const uint32_t cell = (dir_cell(b[1].x) << 4) | (dir_cell(b[1].y) << 2) | dir_cell(b[1].z);
  const uint32_t m = (spread3_6(box_cell(b[0].x, lo.x, scale.x)) << 2) |
                     (spread3_6(box_cell(b[0].y, lo.y, scale.y)) << 1) | spread3_6(box_cell(b[0].z, lo.z, scale.z));
  return min((cell << 18) | m, kMissKey - 1u);
}

// keys[i] = coherence key of ray i's bounce ray (kMissKey for a miss),
// vals[i] = i; *count += the number of hits.
__global__ void __launch_bounds__(256) k_bounce_keys(const float4* __restrict__ rays, const lrt_hit* __restrict__ hits,
                                                     uint64_t n, uint64_t seed, float tnear, float tfar, float3 lo,
                                                     float3 scale, uint32_t* __restrict__ keys,
                                                     uint32_t* __restrict__ vals, unsigned long long* __restrict__ count)
{
  uint32_t c = 0;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const float4 h0 = reinterpret_cast<const float4*>(hits + i)[0];
    uint32_t key = kMissKey;
    if (__float_as_uint(h0.y) != 0xFFFFFFFFu) {
      float4 b[2];
      bounce_ray(rays[2 * i], rays[2 * i + 1], h0, reinterpret_cast<const float4*>(hits + i)[1], i, seed, tnear, tfar,
                 b);
      key = coherence_key(b, lo, scale);
      c++;
    }
    keys[i] = key;
    vals[i] = uint32_t(i);
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

// Bounce ray j of the sorted order: ray index[j]'s, for every j before the
// first miss key (misses sort last, so a thread stops at its first one).
__global__ void __launch_bounds__(256) k_bounce_gather(const float4* __restrict__ rays,
                                                       const lrt_hit* __restrict__ hits, uint64_t n, uint64_t seed,
                                                       float tnear, float tfar, const uint32_t* __restrict__ keys,
                                                       const uint32_t* __restrict__ index, float4* __restrict__ out)
{
  for (uint64_t j = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; j < n; j += uint64_t(gridDim.x) * blockDim.x) {
    if (keys[j] == kMissKey) return;
    const uint64_t i = index[j];
    const float4* h = reinterpret_cast<const float4*>(hits + i);
    bounce_ray(rays[2 * i], rays[2 * i + 1], h[0], h[1], i, seed, tnear, tfar, out + 2 * j);
  }
}

// Arguments shared by the compacting generators.
lrt_status check_compact_args(lrt_scene* s, const char* who, const float* rays_dev, const lrt_hit* hits_dev,
                              const float* bounce_dev, const uint32_t* index_dev, const uint64_t* count_dev)
{
  if (!s) return LRT_ERR_INVALID_ARGUMENT;
  if (!s->dev) return fail(s, LRT_ERR_NOT_COMMITTED, "%s before CommitScene/upload", who);
  if (!rays_dev || !hits_dev || !bounce_dev || !index_dev || !count_dev)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "%s: NULL buffer", who);
  if ((reinterpret_cast<uintptr_t>(rays_dev) | reinterpret_cast<uintptr_t>(hits_dev) |
       reinterpret_cast<uintptr_t>(bounce_dev)) & 15 || (reinterpret_cast<uintptr_t>(count_dev) & 7))
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "%s: misaligned buffer", who);
  return LRT_OK;
}

} // namespace
} // namespace lrt

using namespace lrt;

extern "C" lrt_status lrt_generate_bounce_rays(lrt_scene* s, const float* rays_dev, const lrt_hit* hits_dev, uint64_t n,
                                               uint64_t seed, float tnear, float tfar, float* bounce_dev,
                                               void* stream)
{
  if (!rays_dev || !hits_dev || !bounce_dev)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_generate_bounce_rays: NULL buffer");
  if ((reinterpret_cast<uintptr_t>(rays_dev) | reinterpret_cast<uintptr_t>(hits_dev) |
       reinterpret_cast<uintptr_t>(bounce_dev)) & 15)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_generate_bounce_rays: buffers must be 16-byte aligned");
  if (n == 0) return LRT_OK;
  const int grid = int(std::min<uint64_t>((n + 255) / 256, 148ull * 32));
  k_bounce<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const float4*>(rays_dev), hits_dev, n,
                                                               seed, tnear, tfar, reinterpret_cast<float4*>(bounce_dev));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LRT_OK : (s ? cuda_fail(s, e, "bounce rays") : LRT_ERR_CUDA);
}

extern "C" lrt_status lrt_generate_bounce_rays_compact(lrt_scene* s, const float* rays_dev, const lrt_hit* hits_dev,
                                                       uint64_t n, uint64_t seed, float tnear, float tfar,
                                                       float* bounce_dev, uint32_t* index_dev, uint64_t* count_dev,
                                                       void* stream_p)
{
  lrt_status st = check_compact_args(s, "lrt_generate_bounce_rays_compact", rays_dev, hits_dev, bounce_dev, index_dev,
                                     count_dev);
  if (st != LRT_OK) return st;
  if (n > 0xFFFFFFFFull)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_generate_bounce_rays_compact: more than 2^32 - 1 rays");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  DeviceScene* d = s->dev;
  const uint64_t ntiles = (n + kTile - 1) / kTile;
  if (ntiles > d->tileCap) {
    if (d->tileScratch) cudaFree(d->tileScratch);
    d->tileScratch = nullptr;
    d->tileCap = 0;
    const cudaError_t e = cudaMalloc(&d->tileScratch, std::max<uint64_t>(ntiles, 1) * sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_fail(s, e, "compaction scratch");
    d->tileCap = std::max<uint64_t>(ntiles, 1);
  }
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(count_dev);
  if (n == 0) {
    const cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), stream);
    return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "cudaMemsetAsync");
  }
  k_count_hits<<<uint32_t(ntiles), kCompactThreads, 0, stream>>>(hits_dev, n, d->tileScratch);
  k_scan_tiles<<<1, 1024, 0, stream>>>(d->tileScratch, uint32_t(ntiles), cnt);
  k_bounce_compact<<<uint32_t(ntiles), kCompactThreads, 0, stream>>>(
      reinterpret_cast<const float4*>(rays_dev), hits_dev, n, seed, tnear, tfar, d->tileScratch,
      reinterpret_cast<float4*>(bounce_dev), index_dev);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "bounce compaction");
}

extern "C" lrt_status lrt_generate_bounce_rays_sorted(lrt_scene* s, const float* rays_dev, const lrt_hit* hits_dev,
                                                      uint64_t n, uint64_t seed, float tnear, float tfar,
                                                      float* bounce_dev, uint32_t* index_dev, uint64_t* count_dev,
                                                      void* stream_p)
{
  lrt_status st = check_compact_args(s, "lrt_generate_bounce_rays_sorted", rays_dev, hits_dev, bounce_dev, index_dev,
                                     count_dev);
  if (st != LRT_OK) return st;
  if (n > 0x7FFFFFFFull)
    return fail(s, LRT_ERR_INVALID_ARGUMENT, "lrt_generate_bounce_rays_sorted: more than 2^31 - 1 rays");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  unsigned long long* cnt = reinterpret_cast<unsigned long long*>(count_dev);
  cudaError_t e = cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "cudaMemsetAsync");
  if (n == 0) return LRT_OK;
  // the scene box: the union of the instances' world boxes
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (const lrt_instance_data& in : s->h.instanceData)
    for (int k = 0; k < 3; k++)
      if (in.boxMin[k] <= in.boxMax[k]) {
        lo[k] = std::min(lo[k], in.boxMin[k]);
        hi[k] = std::max(hi[k], in.boxMax[k]);
      }
  float scale[3];
  for (int k = 0; k < 3; k++) {
    const float ext = hi[k] - lo[k];
    scale[k] = (lo[k] <= hi[k] && ext > 0.0f && std::isfinite(ext)) ? 64.0f / ext : 0.0f;
    if (!(lo[k] <= hi[k])) lo[k] = 0.0f;
  }
  DeviceScene* d = s->dev;
  size_t tempBytes = 0;
  e = cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, static_cast<const uint32_t*>(nullptr),
                                      static_cast<uint32_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                      static_cast<uint32_t*>(nullptr), int(n), 0, kKeyBits, stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "radix sort size");
  const size_t words = (3 * n + 63) & ~size_t(63); // keys, sorted keys, ray indices (256-byte aligned)
  const size_t need = words * sizeof(uint32_t) + tempBytes;
  if (need > d->sortBytes) {
    if (d->sortScratch) cudaFree(d->sortScratch);
    d->sortScratch = nullptr;
    d->sortBytes = 0;
    if ((e = cudaMalloc(&d->sortScratch, need)) != cudaSuccess) return cuda_fail(s, e, "bounce sort scratch");
    d->sortBytes = need;
  }
  uint32_t* keys = static_cast<uint32_t*>(d->sortScratch);
  uint32_t* sorted = keys + n;
  uint32_t* vals = keys + 2 * n;
  void* temp = keys + words;
  const int grid = int(std::min<uint64_t>((n + 255) / 256, 148ull * 16));
  const float4* rays = reinterpret_cast<const float4*>(rays_dev);
  k_bounce_keys<<<grid, 256, 0, stream>>>(rays, hits_dev, n, seed, tnear, tfar, make_float3(lo[0], lo[1], lo[2]),
                                          make_float3(scale[0], scale[1], scale[2]), keys, vals, cnt);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(s, e, "bounce keys");
  e = cub::DeviceRadixSort::SortPairs(temp, tempBytes, static_cast<const uint32_t*>(keys), sorted,
                                      static_cast<const uint32_t*>(vals), index_dev, int(n), 0, kKeyBits, stream);
  if (e != cudaSuccess) return cuda_fail(s, e, "radix sort");
  k_bounce_gather<<<grid, 256, 0, stream>>>(rays, hits_dev, n, seed, tnear, tfar, sorted, index_dev,
                                            reinterpret_cast<float4*>(bounce_dev));
  e = cudaGetLastError();
  return e == cudaSuccess ? LRT_OK : cuda_fail(s, e, "bounce gather");
}

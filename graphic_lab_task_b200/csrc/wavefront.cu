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

__global__ void k_bounce(const float4* __restrict__ rays, const lrt_hit* __restrict__ hits, uint64_t n, uint64_t seed,
                         float tnear, float tfar, float4* __restrict__ out)
{
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
    const float4 pn = rays[2 * i], df = rays[2 * i + 1];
    const float4 h0 = reinterpret_cast<const float4*>(hits + i)[0];
    const float4 h1 = reinterpret_cast<const float4*>(hits + i)[1];
    if (__float_as_uint(h0.y) == 0xFFFFFFFFu) {
      const float qnan = __int_as_float(0x7fc00000);
      out[2 * i] = make_float4(qnan, qnan, qnan, tnear);
      out[2 * i + 1] = make_float4(0.0f, 0.0f, 1.0f, tfar);
      continue;
    }
    const f3 dir = mk3(df.x, df.y, df.z);
    const f3 pos = mk3(pn.x, pn.y, pn.z) + h0.x * dir;
    f3 nrm = decode_normal(mk2(h1.z, h1.w));
    if (dot(nrm, dir) > 0.0f) nrm = -1.0f * nrm; // face the incoming ray
    uint64_t state = (i + 1) * 0x9E3779B97F4A7C15ull ^ seed;
    pcg_hash(state);
    const float r1 = uniform01(state), r2 = uniform01(state);
    const f3 b = normalize(cosine_sample(r1, r2, nrm));
    out[2 * i] = make_float4(pos.x, pos.y, pos.z, tnear);
    out[2 * i + 1] = make_float4(b.x, b.y, b.z, tfar);
  }
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

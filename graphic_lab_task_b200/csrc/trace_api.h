// trace_api.h — host launchers exported by trace_exact.cu and trace_fast.cu.
#pragma once
#include <cuda_runtime.h>

#include "device_layout.h"

#define LRT_DECLARE_TRACE_API(NS)                                                                               \
  namespace NS {                                                                                                \
  cudaError_t launch_trace(const lrt::DevScene& S, const float4* rays, lrt_hit* hits, uint64_t n,               \
                           unsigned long long* work_counter, unsigned long long* counters, uint32_t* err_word,  \
                           uint32_t stack_cap, int grid, cudaStream_t stream, bool count, uint32_t img_w = 0,   \
                           uint32_t img_h = 0, const uint32_t* sched_rd = nullptr,                              \
                           uint32_t* sched_wr = nullptr, uint32_t group = 32, bool bricks_only = false);                 \
  cudaError_t set_trace_smem(uint32_t stack_cap);                                                               \
  cudaError_t trace_occupancy(uint32_t stack_cap, int* blocks_per_sm, bool bricks_only = false);                \
  cudaError_t launch_eye_rays(const lrt::DevCamera& cam, float4* rays, cudaStream_t stream);                    \
  cudaError_t launch_trace_cameras(const lrt::DevScene& S, const lrt::DevBatchCamera* cams, uint32_t ncams,     \
                                   uint32_t ntiles, const lrt::DevBatchShape& shape, lrt_hit* hits,             \
                                   unsigned long long* work_counter, uint32_t* err_word, int grid,              \
                                   cudaStream_t stream, const lrt::DevLights* lights = nullptr,                 \
                                   uint32_t* image = nullptr);                                                  \
  cudaError_t cameras_occupancy(uint32_t stack_cap, int* blocks_per_sm);                                        \
  cudaError_t launch_render_rgba8(const lrt::DevScene& S, const lrt::DevCamera& cam, const lrt::DevLights& lights,\
                                  uint32_t* image, unsigned long long* work_counter, uint32_t* err_word,        \
                                  uint32_t stack_cap, int grid, cudaStream_t stream,                            \
                                  const uint32_t* sched_rd = nullptr, uint32_t* sched_wr = nullptr,             \
                                  const lrt::DevMaterials* materials = nullptr,                                 \
                                  const lrt::DevRenderModes* modes = nullptr, bool bricks_only = false);        \
  cudaError_t launch_fill_gbuffer_transparency(const lrt::DevScene& S, const lrt::DevCamera& cam,               \
                                               const lrt::DevMaterials& M, float4* transparency, lrt_hit* gbuffer,\
                                               unsigned long long* work_counter, uint32_t* err_word,            \
                                               uint32_t stack_cap, int grid, cudaStream_t stream,               \
                                               const uint32_t* sched_rd = nullptr,                              \
                                               uint32_t* sched_wr = nullptr);                                   \
  cudaError_t launch_outline_fill(const lrt::DevScene& S, const lrt::DevCamera& cam, const lrt::DevLights& lights, \
                                 const lrt::DevMaterials& M, const lrt::DevRenderModes& RM, uint32_t smp,       \
                                 float2* tm, float4* col, unsigned long long* work_counter, uint32_t* err_word, \
                                 uint32_t stack_cap, int grid, cudaStream_t stream, const uint32_t* sched_rd,   \
                                 uint32_t* sched_wr);                                                           \
  cudaError_t launch_outline_resolve(const float2* tm, const float4* col, uint32_t w, uint32_t h, uint32_t smp,  \
                                     uint32_t samples, float4* acc, uint32_t* image, cudaStream_t stream);     \
  cudaError_t launch_render_lambert(const lrt::DevScene& S, const float4* rays, uint64_t n, float3 light,       \
                                    float* image, unsigned long long* work_counter, uint32_t* err_word,         \
                                    uint32_t stack_cap, int grid, cudaStream_t stream, uint32_t img_w = 0,      \
                                    uint32_t img_h = 0, const uint32_t* sched_rd = nullptr,                     \
                                    uint32_t* sched_wr = nullptr);                                              \
  cudaError_t launch_adjoint_lambert(const lrt::DevScene& S, const float4* rays, uint64_t n, float3 light,      \
                                     const float* dimage, float* grad, unsigned long long* work_counter,        \
                                     uint32_t* err_word, uint32_t stack_cap, int grid, cudaStream_t stream,     \
                                     uint32_t img_w = 0, uint32_t img_h = 0, const uint32_t* sched_rd = nullptr, \
                                     uint32_t* sched_wr = nullptr);                                             \
  }

LRT_DECLARE_TRACE_API(lrt_exact)
LRT_DECLARE_TRACE_API(lrt_fast)

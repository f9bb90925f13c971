// lrt_math.h — scalar float3 helpers shared by host C++ and sm_100a device code.
//
// Every helper evaluates in the operation order of the reference's LiteMath
// (dependencies/1st-party/LiteMath/LiteMath.h) so that, compiled without
// FMA contraction (-ffp-contract=off on the host, -fmad=false on the device),
// host and device produce identical bits.  std::min/std::max semantics
// ((b < a) ? b : a and (a < b) ? b : a) are kept literally: they differ from
// fminf/fmaxf on NaN, and NaNs do occur for axis-parallel rays.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define LRT_HD __host__ __device__ __forceinline__
#else
#define LRT_HD inline
#endif

namespace lrt {

struct f3 {
  float x, y, z;
};
struct f2 {
  float x, y;
};

LRT_HD f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
LRT_HD f2 mk2(float x, float y) { f2 r; r.x = x; r.y = y; return r; }
LRT_HD f3 operator+(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
LRT_HD f3 operator-(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
LRT_HD f3 operator*(f3 a, f3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
LRT_HD f3 operator*(float s, f3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
LRT_HD f3 operator*(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
LRT_HD f3 operator/(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }

LRT_HD float smin(float a, float b) { return (b < a) ? b : a; }   // std::min
LRT_HD float smax(float a, float b) { return (a < b) ? b : a; }   // std::max
LRT_HD float sclamp(float u, float a, float b) { return smin(smax(a, u), b); } // LiteMath clamp
// LiteMath clamp for bounds 0 < a <= b: equal to fminf(fmaxf(u, a), b) for
// every u (a NaN u gives a in both forms; a zero u of either sign gives a).
LRT_HD float sclamp_pos(float u, float a, float b) { return fminf(fmaxf(u, a), b); }
LRT_HD float ssign(float x) { return x == 0.0f ? 0.0f : (x < 0.0f ? -1.0f : 1.0f); } // LiteMath.h:133-138

LRT_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// LiteMath cross (LiteMath.h:987-992): shuffle_yzx(a*b_yzx - a_yzx*b)
LRT_HD f3 cross(f3 a, f3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
// LiteMath normalize: v * (1/sqrt(dot(v,v)))
LRT_HD f3 normalize(f3 v)
{
  const float inv = 1.0f / sqrtf(dot(v, v));
  return mk3(v.x * inv, v.y * inv, v.z * inv);
}

// column-major float4x4 * float4 (mat4_colmajor_mul_vec4, LiteMath.h:1813-1819),
// returning xyz; w=1 is matmul4x3, w=0 is matmul3x3 (raytrace_common.h:85-93).
LRT_HD f3 matmul4(const float* m, f3 v, float w)
{
  f3 r;
  r.x = v.x * m[0] + v.y * m[4] + v.z * m[8] + w * m[12];
  r.y = v.x * m[1] + v.y * m[5] + v.z * m[9] + w * m[13];
  r.z = v.x * m[2] + v.y * m[6] + v.z * m[10] + w * m[14];
  return r;
}

// SafeInverse, utils/raytracing/raytrace_common.h:59-67
LRT_HD f3 safe_inverse(f3 d)
{
  const float ooeps = 1.0e-36f;
  f3 r;
  r.x = 1.0f / (fabsf(d.x) > ooeps ? d.x : fabsf(ooeps) * ssign(d.x));
  r.y = 1.0f / (fabsf(d.y) > ooeps ? d.y : fabsf(ooeps) * ssign(d.y));
  r.z = 1.0f / (fabsf(d.z) > ooeps ? d.z : fabsf(ooeps) * ssign(d.z));
  return r;
}

// RayBoxIntersection2, utils/raytracing/raytrace_common.h:69-82
LRT_HD f2 ray_box(f3 o, f3 inv, f3 bmin, f3 bmax)
{
  const float lo = inv.x * (bmin.x - o.x);
  const float hi = inv.x * (bmax.x - o.x);
  const float lo1 = inv.y * (bmin.y - o.y);
  const float hi1 = inv.y * (bmax.y - o.y);
  const float lo2 = inv.z * (bmin.z - o.z);
  const float hi2 = inv.z * (bmax.z - o.z);
  const float tmin = smax(smin(lo, hi), smin(lo1, hi1));
  const float tmax = smin(smax(lo, hi), smax(lo1, hi1));
  return mk2(smax(tmin, smin(lo2, hi2)), smin(tmax, smax(lo2, hi2)));
}

// RayBoxIntersection2 with one-instruction min/max, for node tests only.
// std::min/max differ from fminf/fmaxf only when an operand is NaN (and in
// which zero they return for +0/-0).  A slab value inv*(b - o) is NaN only if
// an inverse-direction component is infinite (SafeInverse of an exactly zero
// component), so for rays with a finite inverse this returns the same
// interval up to the sign of zeros — and node tests only compare the
// interval ends (<=, <, >), where +0 == -0.  The caller checks finiteness.
LRT_HD f2 ray_box_nodes(f3 o, f3 inv, f3 bmin, f3 bmax)
{
  const float lo = inv.x * (bmin.x - o.x);
  const float hi = inv.x * (bmax.x - o.x);
  const float lo1 = inv.y * (bmin.y - o.y);
  const float hi1 = inv.y * (bmax.y - o.y);
  const float lo2 = inv.z * (bmin.z - o.z);
  const float hi2 = inv.z * (bmax.z - o.z);
  const float tmin = fmaxf(fminf(lo, hi), fminf(lo1, hi1));
  const float tmax = fminf(fmaxf(lo, hi), fmaxf(lo1, hi1));
  return mk2(fmaxf(tmin, fminf(lo2, hi2)), fminf(tmax, fmaxf(lo2, hi2)));
}

LRT_HD bool finite3(f3 v) { return fabsf(v.x) < INFINITY && fabsf(v.y) < INFINITY && fabsf(v.z) < INFINITY; }

// The six slab values of RayBoxIntersection2, and its two results computed
// from them separately (near = .x, far = .y of ray_box), in the literal
// std::min/max form or (FAST) the one-instruction form.  For a finite box
// and a ray with finite origin, direction and inverse no slab value is NaN,
// so the two forms give the same numbers up to the sign of a zero result.
struct Slabs {
  float lo, hi, lo1, hi1, lo2, hi2;
};

LRT_HD Slabs slabs(f3 o, f3 inv, f3 bmin, f3 bmax)
{
  Slabs s;
  s.lo = inv.x * (bmin.x - o.x);
  s.hi = inv.x * (bmax.x - o.x);
  s.lo1 = inv.y * (bmin.y - o.y);
  s.hi1 = inv.y * (bmax.y - o.y);
  s.lo2 = inv.z * (bmin.z - o.z);
  s.hi2 = inv.z * (bmax.z - o.z);
  return s;
}

template <bool FAST>
LRT_HD float slab_near(const Slabs& s)
{
  if (FAST) return fmaxf(fmaxf(fminf(s.lo, s.hi), fminf(s.lo1, s.hi1)), fminf(s.lo2, s.hi2));
  return smax(smax(smin(s.lo, s.hi), smin(s.lo1, s.hi1)), smin(s.lo2, s.hi2));
}

template <bool FAST>
LRT_HD float slab_far(const Slabs& s)
{
  if (FAST) return fminf(fminf(fmaxf(s.lo, s.hi), fmaxf(s.lo1, s.hi1)), fmaxf(s.lo2, s.hi2));
  return smin(smin(smax(s.lo, s.hi), smax(s.lo1, s.hi1)), smax(s.lo2, s.hi2));
}

// encode_normal, utils/raytracing/intersection_common.h:96-101 (octahedral)
LRT_HD f2 encode_normal(f3 v)
{
  const float inv = 1.0f / (fabsf(v.x) + fabsf(v.y) + fabsf(v.z));
  const f2 p = mk2(v.x * inv, v.y * inv);
  const float sx = (p.x >= 0.0f) ? 1.0f : -1.0f;
  const float sy = (p.y >= 0.0f) ? 1.0f : -1.0f;
  return (v.z <= 0.0f) ? mk2((1.0f - fabsf(p.y)) * sx, (1.0f - fabsf(p.x)) * sy) : p;
}

// decode_normal, utils/raytracing/render_common.h:257-266
LRT_HD f3 decode_normal(f2 e)
{
  f3 v = mk3(e.x, e.y, 1.0f - fabsf(e.x) - fabsf(e.y));
  if (v.z < 0) {
    const float vx = v.x;
    v.x = (1.0f - fabsf(v.y)) * ((v.x >= 0.0f) ? +1.0f : -1.0f);
    v.y = (1.0f - fabsf(vx)) * ((v.y >= 0.0f) ? +1.0f : -1.0f);
  }
  return normalize(v);
}

// eval_dist_trilinear, MultiRenderer/BVH2Common.cpp:126-136
// corner order 000,001,010,011,100,101,110,111 with x the most significant bit.
LRT_HD float trilinear(const float* v, f3 dp)
{
  return (1 - dp.x) * (1 - dp.y) * (1 - dp.z) * v[0] + (1 - dp.x) * (1 - dp.y) * (dp.z) * v[1] +
         (1 - dp.x) * (dp.y) * (1 - dp.z) * v[2] + (1 - dp.x) * (dp.y) * (dp.z) * v[3] +
         (dp.x) * (1 - dp.y) * (1 - dp.z) * v[4] + (dp.x) * (1 - dp.y) * (dp.z) * v[5] +
         (dp.x) * (dp.y) * (1 - dp.z) * v[6] + (dp.x) * (dp.y) * (dp.z) * v[7];
}

// MultiRenderer::initEyeRay (MultiRenderer.cpp:142-183) for spp = 1, frame 0,
// cutting plane disabled: EyeRayDirNormalized + transform_ray3f
// (utils/raytracing/render_common.h:25-55).  out = {posAndNear, dirAndFar}.
LRT_HD void eye_ray(const float* proj_inv, const float* world_view_inv, uint32_t x, uint32_t y, uint32_t w,
                    uint32_t h, float tnear, float tfar, float* out, float dx = 0.5f, float dy = 0.5f)
{
  // (dx, dy): the sample's position in the pixel (initEyeRay's d)
  const float fx = ((float)x + dx) / (float)w;
  const float fy = ((float)y + dy) / (float)h;
  const float px = 2.0f * fx - 1.0f, py = -2.0f * fy + 1.0f;
  // pos = projInv * float4(px, py, 1, 1); pos /= pos.w
  float q[4];
  for (int i = 0; i < 4; i++)
    q[i] = px * proj_inv[i] + py * proj_inv[4 + i] + 1.0f * proj_inv[8 + i] + 1.0f * proj_inv[12 + i];
  const float qw = q[3];
  f3 dir = normalize(mk3(q[0] / qw, q[1] / qw, q[2] / qw));
  const f3 zero = mk3(0.0f, 0.0f, 0.0f);
  const f3 pos = matmul4(world_view_inv, zero, 1.0f);
  const f3 pos2 = matmul4(world_view_inv, zero + 100.0f * dir, 1.0f);
  dir = normalize(pos2 - pos);
  out[0] = pos.x; out[1] = pos.y; out[2] = pos.z; out[3] = tnear;
  out[4] = dir.x; out[5] = dir.y; out[6] = dir.z; out[7] = tfar;
}

} // namespace lrt

/*
 * lrt_oracle.c — CPU restatement of LiteRT's nearest-hit ray query.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 * The product library never links or calls it.
 *
 * It restates, in plain C with IEEE single-precision arithmetic evaluated in
 * the reference's operation order (build with -ffp-contract=off), the path
 *   BVHRT::RayQuery_NearestHit   MultiRenderer/BVH2Common.cpp:3322-3392
 *   BVHRT::BVH2TraverseF32       MultiRenderer/BVH2Common.cpp:3239-3320
 *   IntersectAllPrimitivesInLeaf MultiRenderer/BVH2Common.cpp:47-124
 *   IntersectAllTrianglesInLeaf  MultiRenderer/BVH2Common.cpp:1571-1635
 *   OctreeNodeIntersect / RayNodeIntersection  :727-749, :141-218
 *   OctreeBrickIntersect / load_distance_values :884-1112, :846-882
 *   LocalSurfaceIntersection (ST branch)        :345-391, :618-690
 * over the flattened BVHRT arrays (lrt_scene_arrays).  Its results are
 * pinned against the reference compiled from its own sources (oracle/ref)
 * and against committed golden vectors (tests/golden).
 *
 * Differences from the reference, all on inputs where the reference is
 * undefined: the BLAS stack is checked against its 80-entry capacity
 * (raytrace_common.h:36 has no check), the SBS voxel march is capped at
 * LRTO_MAX_VOXEL_STEPS iterations (the reference loop can stall when
 * t + 1e-6 rounds back to t), and out-of-range node ids end the leaf test.
 * Each such event increments the `limits` counter instead.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/lrt_b200.h"

#define LEAF_BIT 0x80000000u
#define START_MASK 0x0FFFFFFFu
#define SIZE_MASK 0x70000000u
#define STACK_SIZE 80
#define LRTO_MAX_VOXEL_STEPS 4096u

enum {
  C_TLAS_NODES = 0, C_INSTANCES, C_BLAS_PAIRS, C_LEAF_CALLS, C_TRI_TESTS, C_BRICKS, C_VOXELS, C_ST_STEPS,
  C_OCTREE_LEAVES, C_SVS_LEAVES, C_HITS, C_NORMALS, C_VOXEL_LOADS
};

typedef struct { float x, y, z; } f3;
typedef struct { float x, y; } f2;

/* std::min / std::max / LiteMath::clamp / LiteMath::sign, in their exact
 * comparison forms (NaN propagation matters for bit parity). */
static inline float smin(float a, float b) { return (b < a) ? b : a; }
static inline float smax(float a, float b) { return (a < b) ? b : a; }
static inline float sclamp(float u, float a, float b) { return smin(smax(a, u), b); }
#define LRT_PI_F 3.14159265358979323846f /* LiteMath::M_PI, a float (LiteMath.h:60) */
static inline float ssign(float x) { return x == 0.0f ? 0.0f : (x < 0.0f ? -1.0f : 1.0f); }

static inline f3 mk3(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 add3(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 sub3(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 mul3(f3 a, f3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline f3 scl3(float s, f3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
static inline f3 div3s(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
static inline float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* LiteMath cross (LiteMath.h:987-992) */
static inline f3 cross3(f3 a, f3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
/* LiteMath normalize: v * (1/sqrt(dot(v,v))) (LiteMath.h:966) */
static inline f3 normalize3(f3 v) { float inv = 1.0f / sqrtf(dot3(v, v)); return mk3(v.x * inv, v.y * inv, v.z * inv); }
static inline f3 ld3(const float* p) { return mk3(p[0], p[1], p[2]); }

/* float4x4 (column-major) times float4, mat4_colmajor_mul_vec4
 * (LiteMath.h:1813-1819); matmul4x3 uses w=1, matmul3x3 w=0
 * (raytrace_common.h:85-93). */
static inline f3 matmul4(const float* m, f3 v, float w)
{
  f3 r;
  r.x = v.x * m[0] + v.y * m[4] + v.z * m[8] + w * m[12];
  r.y = v.x * m[1] + v.y * m[5] + v.z * m[9] + w * m[13];
  r.z = v.x * m[2] + v.y * m[6] + v.z * m[10] + w * m[14];
  return r;
}

/* SafeInverse, raytrace_common.h:59-67 */
static inline f3 safe_inverse(f3 d)
{
  const float ooeps = 1.0e-36f;
  f3 r;
  r.x = 1.0f / (fabsf(d.x) > ooeps ? d.x : fabsf(ooeps) * ssign(d.x));
  r.y = 1.0f / (fabsf(d.y) > ooeps ? d.y : fabsf(ooeps) * ssign(d.y));
  r.z = 1.0f / (fabsf(d.z) > ooeps ? d.z : fabsf(ooeps) * ssign(d.z));
  return r;
}

/* RayBoxIntersection2, raytrace_common.h:69-82 */
static inline f2 ray_box(f3 o, f3 inv, f3 bmin, f3 bmax)
{
  const float lo = inv.x * (bmin.x - o.x);
  const float hi = inv.x * (bmax.x - o.x);
  const float lo1 = inv.y * (bmin.y - o.y);
  const float hi1 = inv.y * (bmax.y - o.y);
  const float lo2 = inv.z * (bmin.z - o.z);
  const float hi2 = inv.z * (bmax.z - o.z);
  const float tmin = smax(smin(lo, hi), smin(lo1, hi1));
  const float tmax = smin(smax(lo, hi), smax(lo1, hi1));
  f2 r = {smax(tmin, smin(lo2, hi2)), smin(tmax, smax(lo2, hi2))};
  return r;
}

/* encode_normal, intersection_common.h:96-101 */
static inline f2 encode_normal(f3 v)
{
  const float inv = 1.0f / (fabsf(v.x) + fabsf(v.y) + fabsf(v.z));
  f2 p = {v.x * inv, v.y * inv};
  const float sx = (p.x >= 0.0f) ? 1.0f : -1.0f;
  const float sy = (p.y >= 0.0f) ? 1.0f : -1.0f;
  if (v.z <= 0.0f) {
    f2 r = {(1.0f - fabsf(p.y)) * sx, (1.0f - fabsf(p.x)) * sy};
    return r;
  }
  return p;
}

/* eval_dist_trilinear, BVH2Common.cpp:126-136 */
static inline float trilinear(const float v[8], f3 dp)
{
  return (1 - dp.x) * (1 - dp.y) * (1 - dp.z) * v[0] + (1 - dp.x) * (1 - dp.y) * (dp.z) * v[1] +
         (1 - dp.x) * (dp.y) * (1 - dp.z) * v[2] + (1 - dp.x) * (dp.y) * (dp.z) * v[3] +
         (dp.x) * (1 - dp.y) * (1 - dp.z) * v[4] + (dp.x) * (1 - dp.y) * (dp.z) * v[5] +
         (dp.x) * (dp.y) * (1 - dp.z) * v[6] + (dp.x) * (dp.y) * (dp.z) * v[7];
}

/* The hit voxel of an SBS hit, recorded for the adjoint (project-written:
 * the reference has no differentiable renderer). */
typedef struct {
  float t;
  float values[8];
  uint32_t idx[8];
  f3 p, dir;
  float d;
  int sbs;
  int early; /* hit at the voxel entry (field already <= EPS there): fixed point */
} hit_record_t;

typedef struct {
  const lrt_scene_arrays* a;
  const lrt_preset* p;
  uint64_t* cnt;   /* LRT_COUNTER_COUNT entries (thread-local) */
  uint64_t limits; /* bounded-loop / bounds events */
  hit_record_t* rec; /* NULL unless recording */
  uint32_t tri_local; /* a triangle hit's primId before the m_primIndices remap */
} ctx_t;

/* BVHRT::need_normal, BVH2Common.cpp:19-32 */
static int need_normal(const lrt_preset* p)
{
  const uint32_t m = p->render_mode;
  return m == 1 || m == 8 || m == 12 || m == 17 || m == 20 || m == 7 || m == 18 || m == 23 || m == 21 ||
         m == 11 || m == 27;
}

/* The cubic c3 t^3 + c2 t^2 + c1 t + c0 whose root is the trilinear
 * surface along the ray inside one voxel, in voxel units (BVH2Common.cpp:395-436,
 * after "Ray Tracing of Signed Distance Function Grids", JCGT 11(3), 2022). */
static void sdf_cubic(const float values[8], float d_inv, f3 o, f3 d3, float c[4])
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

/* ANALYTIC: the smallest non-negative real root of the cubic (Vieta /
 * Cardano for a cubic, the stable quadratic formula, the linear root),
 * roots below 0 replaced by 1000 (BVH2Common.cpp:441-505).  The reference's
 * unqualified sqrt there is the C library's double sqrt, so the expressions
 * that contain it are evaluated in double and rounded to float on
 * assignment; std::sqrt, std::cos of a float and M_PI (LiteMath's float)
 * stay in float. */
static float sdf_root_analytic(const float c[4], float EPS)
{
  const float c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
  float x1 = 1000, x2 = 1000, x3 = 1000;
  if (fabsf(c3) > 1e-5f) {
    const float a = c2 / c3, b = c1 / c3, cc = c0 / c3;
    const float Q = (a * a - 3 * b) / 9;
    const float R = (2 * a * a * a - 9 * a * b + 27 * cc) / 54;
    const float Q3 = Q * Q * Q;
    if (R * R < Q3) {
      const float theta = (float)acos(R / sqrt(Q3));
      x1 = (float)(-2 * sqrt(Q) * cosf(theta / 3) - a / 3);
      x2 = (float)(-2 * sqrt(Q) * cosf((theta + 2 * LRT_PI_F) / 3) - a / 3);
      x3 = (float)(-2 * sqrt(Q) * cosf((theta - 2 * LRT_PI_F) / 3) - a / 3);
    } else {
      const float A = (float)(-ssign(R) * pow(fabsf(R) + sqrt(R * R - Q3), 1.0f / 3.0f));
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

/* NEWTON: bracket a sign change of the cubic between 0, the roots of its
 * derivative and qFar, then at most 10 Newton steps from the middle of the
 * bracket (BVH2Common.cpp:507-587).  Returns the hit flag; *t the root. */
static int sdf_root_newton(const float c[4], float qFar, float EPS, float* t)
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
  const int s0 = c0 > 0;
  const int s1 = (c0 + t1 * (c1 + t1 * (c2 + t1 * c3))) > 0;
  const int s2 = (c0 + t2 * (c1 + t2 * (c2 + t2 * c3))) > 0;
  const int s3 = (c0 + t3 * (c1 + t3 * (c2 + t3 * c3))) > 0;
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
  if (!(nwt_min < nwt_max)) return 0;
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
  *t = rtn;
  return rtn >= 0 && rtn <= qFar && fabsf(f) < EPS;
}

/* LocalSurfaceIntersection, trilinear (BVH2Common.cpp:345-690): the ST,
 * BBOX, ANALYTIC, NEWTON and IT node solvers.  is_surface_node is always
 * false on this path (OctreeNodeIntersect and OctreeBrickIntersect pass
 * false), so EPS is the base 1e-6. */
static void local_surface(ctx_t* c, uint32_t type, f3 ray_dir, uint32_t instId, uint32_t geomId,
                          const float values[8], uint32_t primId, float d, float qNear, float qFar, f2 fNearFar,
                          f3 start_q, lrt_hit* hit)
{
  const lrt_preset* P = c->p;
  const float EPS = 1e-6f;
  const float d_inv = 1.0f / d;
  float t = qNear;
  int early_hit = 0, hitf = 0;
  unsigned iter = 0;
  float start_sign = 1;
  float start_dist = trilinear(values, add3(start_q, scl3(t, ray_dir)));
  c->cnt[C_ST_STEPS]++;
  if (P->representation_mode == 0 /* SURFACE */) start_sign = ssign(start_dist);
  start_dist *= start_sign;
  if (start_dist <= EPS || P->sdf_node_intersect == 3 /* BBOX */) {
    early_hit = 1;
    hitf = 1;
  } else if (P->sdf_node_intersect == 0 /* ST */) {
    float dist = start_dist;
    while (t < qFar && dist > EPS && iter < 256) {
      t += dist * d_inv;
      dist = start_sign * trilinear(values, add3(start_q, scl3(t, ray_dir)));
      iter++;
    }
    c->cnt[C_ST_STEPS] += iter;
    hitf = (dist <= EPS);
  } else {
    float cf[4];
    sdf_cubic(values, d_inv, start_q, ray_dir, cf);
    if (P->sdf_node_intersect == 1 /* ANALYTIC */) {
      t = sdf_root_analytic(cf, EPS);
      hitf = (t >= 0 && t <= qFar);
    } else if (P->sdf_node_intersect == 2 /* NEWTON */) {
      hitf = sdf_root_newton(cf, qFar, EPS, &t);
    } else { /* IT: interval tracing with the cubic's derivative as a Lipschitz bound (:588-618) */
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
        dist = start_sign * trilinear(values, add3(start_q, scl3(t, ray_dir)));
        iter++;
      }
      c->cnt[C_ST_STEPS] += iter;
      hitf = (dist <= EPS);
    }
  }
  const float tReal = fNearFar.x + d * t;
  if (t <= qFar && hitf && tReal < hit->t) {
    f3 norm = mk3(0, 0, 1);
    if (need_normal(P)) {
      const lrt_instance_data* inst = &c->a->instanceData[instId];
      if (early_hit && P->sdf_node_intersect == 3) {
        /* BVH2Common.cpp:644-656 */
        float q[3] = {start_q.x, start_q.y, start_q.z};
        f3 v = mk3(smax(start_q.x, 1 - start_q.x), smax(start_q.y, 1 - start_q.y), smax(start_q.z, 1 - start_q.z));
        int dim = 0;
        if (v.y > v.x && v.y > v.z) dim = 1;
        else if (v.z > v.x && v.z > v.y) dim = 2;
        float n[3] = {0, 0, 0};
        n[dim] = q[dim] < 0.5f ? -1.0f : 1.0f;
        norm = mk3(n[0], n[1], n[2]);
      } else {
        /* qNear is 0 on this path, so the cutting-plane branch (:640-643) is unreachable */
        const f3 p0 = add3(start_q, scl3(t, ray_dir));
        const float h = 0.001f;
        float ddx = (trilinear(values, add3(p0, mk3(h, 0, 0))) - trilinear(values, add3(p0, mk3(-h, 0, 0)))) / (2 * h);
        float ddy = (trilinear(values, add3(p0, mk3(0, h, 0))) - trilinear(values, add3(p0, mk3(0, -h, 0)))) / (2 * h);
        float ddz = (trilinear(values, add3(p0, mk3(0, 0, h))) - trilinear(values, add3(p0, mk3(0, 0, -h)))) / (2 * h);
        norm = scl3(start_sign, mk3(ddx, ddy, ddz));
      }
      norm = normalize3(matmul4(inst->transformInvTransposed, norm, 1.0f));
      c->cnt[C_NORMALS]++;
    }
    const f2 en = encode_normal(norm);
    if (c->rec) {
      c->rec->t = tReal;
      for (int i = 0; i < 8; i++) c->rec->values[i] = values[i];
      c->rec->p = add3(start_q, scl3(t, ray_dir));
      c->rec->dir = ray_dir;
      c->rec->d = d;
      c->rec->sbs = 0;
      c->rec->early = early_hit;
    }
    hit->t = tReal;
    hit->primId = primId;
    hit->instId = instId;
    hit->geomId = geomId | (type << 24);
    hit->coords[0] = 0;
    hit->coords[1] = 0;
    hit->coords[2] = en.x;
    hit->coords[3] = en.y;
    if (P->render_mode == LRT_RENDER_MODE_ST_ITERATIONS) hit->primId = iter;
  }
}

/* OctreeNodeIntersect + RayNodeIntersection (BVH2Common.cpp:727-749, 141-218). */
static void octree_node(ctx_t* c, uint32_t type, f3 ray_pos, f3 ray_dir, float tNear, uint32_t instId,
                        uint32_t geomId, uint32_t bvhNodeId, lrt_hit* hit)
{
  const lrt_scene_arrays* A = c->a;
  float values[8];
  uint32_t primId;
  f3 min_pos, max_pos;
  const uint32_t sdfId = A->geomData[geomId].offset[0];
  if (type == LRT_TYPE_SDF_FRAME_OCTREE) {
    c->cnt[C_OCTREE_LEAVES]++;
    if (bvhNodeId >= A->origNodes_count) { c->limits++; return; }
    const lrt_bvh_node* on = &A->origNodes[bvhNodeId];
    primId = on->leftOffset;
    const uint64_t nodeId = (uint64_t)primId + A->sdfFrameOctreeRoots[sdfId];
    if (nodeId >= A->sdfFrameOctreeNodes_count) { c->limits++; return; }
    min_pos = ld3(on->boxMin);
    max_pos = ld3(on->boxMax);
    for (int i = 0; i < 8; i++) values[i] = A->sdfFrameOctreeNodes[nodeId].values[i];
  } else if (type == LRT_TYPE_SDF_SVS) {
    c->cnt[C_SVS_LEAVES]++;
    primId = bvhNodeId;
    const uint64_t nodeId = (uint64_t)primId + A->sdfSVSRoots[sdfId];
    if (nodeId >= A->sdfSVSNodes_count) { c->limits++; return; }
    const lrt_sdf_svs_node* n = &A->sdfSVSNodes[nodeId];
    const float px = (float)(n->pos_xy >> 16);
    const float py = (float)(n->pos_xy & 0x0000FFFF);
    const float pz = (float)(n->pos_z_lod_size >> 16);
    const float sz = (float)(n->pos_z_lod_size & 0x0000FFFF);
    const float d_max = 2 * 1.73205081f / sz;
    min_pos = add3(mk3(-1, -1, -1), div3s(scl3(2.0f, mk3(px, py, pz)), sz));
    max_pos = add3(min_pos, div3s(scl3(2.0f, mk3(1, 1, 1)), sz));
    for (int i = 0; i < 8; i++)
      values[i] = -d_max + 2.0f * d_max * (1.0f / 255.0f) * ((n->values[i / 4] >> (8 * (i % 4))) & 0xFF);
  } else {
    return;
  }
  const f3 size = sub3(max_pos, min_pos);
  const f2 fNearFar = ray_box(ray_pos, safe_inverse(ray_dir), min_pos, max_pos);
  const f3 start_pos = add3(ray_pos, scl3(fNearFar.x, ray_dir));
  const float d = smax(size.x, smax(size.y, size.z));
  const f3 start_q = div3s(sub3(start_pos, min_pos), d);
  const float qFar = (fNearFar.y - fNearFar.x) / d;
  const float qNear = tNear > fNearFar.x ? (tNear - fNearFar.x) / d : 0.0f;
  if (qNear > 0.0f) return; /* ray starts inside this node (:744-745) */
  local_surface(c, type, ray_dir, instId, geomId, values, primId, d, qNear, qFar, fNearFar, start_q, hit);
}

/* load_distance_values, BVH2Common.cpp:846-882 (trilinear corners 000..111, x major). */
static float load_distance_values(ctx_t* c, uint32_t nodeId, f3 voxelPos, uint32_t v_size, float sz_inv,
                                  const lrt_sdf_sbs_header* h, float values[8])
{
  const lrt_scene_arrays* A = c->a;
  float vmin = 1e6f;
  const uint32_t v_off = A->sdfSBSNodes[nodeId].data_offset;
  const uint32_t layout = h->aux_data & LRT_SBS_LAYOUT_MASK;
  const uint32_t vx = (uint32_t)voxelPos.x, vy = (uint32_t)voxelPos.y, vz = (uint32_t)voxelPos.z;
  if (layout == LRT_SBS_LAYOUT_ID32F_IRGB32F || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN) {
    for (int i = 0; i < 8; i++) {
      const uint32_t x = vx + ((i & 4) >> 2), y = vy + ((i & 2) >> 1), z = vz + (i & 1);
      const uint32_t vId = (x + h->brick_pad) * v_size * v_size + (y + h->brick_pad) * v_size + (z + h->brick_pad);
      values[i] = A->sdfSBSDataF[A->sdfSBSData[v_off + vId]];
      vmin = smin(vmin, values[i]);
    }
  } else {
    const uint32_t vals_per_int = 4 / h->bytes_per_value;
    const uint32_t bits = 8 * h->bytes_per_value;
    const uint32_t max_val = h->bytes_per_value == 4 ? 0xFFFFFFFFu : ((1u << bits) - 1);
    const float d_max = 1.73205081f * sz_inv;
    const float mult = 2 * d_max / max_val;
    for (int i = 0; i < 8; i++) {
      const uint32_t x = vx + ((i & 4) >> 2), y = vy + ((i & 2) >> 1), z = vz + (i & 1);
      const uint32_t vId = (x + h->brick_pad) * v_size * v_size + (y + h->brick_pad) * v_size + (z + h->brick_pad);
      const uint32_t word = A->sdfSBSData[v_off + vId / vals_per_int];
      const uint32_t sh = bits * (vId % vals_per_int);
      const uint32_t field = (sh >= 32 ? 0u : (word >> sh)) & max_val;
      values[i] = -d_max + mult * field;
      vmin = smin(vmin, values[i]);
    }
  }
  return vmin;
}

/* OctreeBrickIntersect, trilinear, BVH2Common.cpp:884-1112 (SMOOTHED normals
 * and tricubic filtering are outside the path). */
static void octree_brick(ctx_t* c, uint32_t type, f3 ray_pos, f3 ray_dir, float tNear, uint32_t instId,
                         uint32_t geomId, uint32_t bvhNodeId, lrt_hit* hit)
{
  const lrt_scene_arrays* A = c->a;
  const uint32_t sdfId = A->geomData[geomId].offset[0];
  const uint32_t primId = bvhNodeId;
  const uint64_t nodeId64 = (uint64_t)primId + A->sdfSBSRoots[sdfId];
  c->cnt[C_BRICKS]++;
  if (nodeId64 >= A->sdfSBSNodes_count) { c->limits++; return; }
  const uint32_t nodeId = (uint32_t)nodeId64;
  const lrt_sdf_sbs_header h = A->sdfSBSHeaders[sdfId];
  const uint32_t v_size = h.brick_size + 2 * h.brick_pad + 1;
  const lrt_sdf_sbs_node* n = &A->sdfSBSNodes[nodeId];
  const float px = (float)(n->pos_xy >> 16);
  const float py = (float)(n->pos_xy & 0x0000FFFF);
  const float pz = (float)(n->pos_z_lod_size >> 16);
  const float sz = (float)(n->pos_z_lod_size & 0x0000FFFF);
  const float sz_inv = 2.0f / sz;
  const float d = 2.0f / (sz * h.brick_size);
  const f3 brick_min_pos = add3(mk3(-1, -1, -1), scl3(sz_inv, mk3(px, py, pz)));
  const f3 brick_max_pos = add3(brick_min_pos, scl3(sz_inv, mk3(1, 1, 1)));
  const f3 inv_dir = safe_inverse(ray_dir);
  f2 bnf = ray_box(ray_pos, inv_dir, brick_min_pos, brick_max_pos);
  const float old_t = hit->t;
  const float scale = 0.5f * sz * h.brick_size;
  float values[8];
  uint32_t steps = 0;
  while (bnf.x < bnf.y && hit->t == old_t) {
    if (steps++ >= LRTO_MAX_VOXEL_STEPS) { c->limits++; break; }
    c->cnt[C_VOXELS]++;
    const f3 hit_pos = add3(ray_pos, scl3(bnf.x, ray_dir));
    const f3 local_pos = scl3(scale, sub3(hit_pos, brick_min_pos));
    const float hi = h.brick_size - 1e-6f;
    const f3 voxelPos = mk3(floorf(sclamp(local_pos.x, 1e-6f, hi)), floorf(sclamp(local_pos.y, 1e-6f, hi)),
                            floorf(sclamp(local_pos.z, 1e-6f, hi)));
    const f3 min_pos = add3(brick_min_pos, scl3(d, voxelPos));
    const f3 max_pos = add3(min_pos, scl3(d, mk3(1, 1, 1)));
    const float vmin = load_distance_values(c, nodeId, voxelPos, v_size, sz_inv, &h, values);
    const f2 fNearFar = ray_box(ray_pos, inv_dir, min_pos, max_pos);
    if (tNear < fNearFar.x && vmin <= 0.0f) {
      c->cnt[C_VOXEL_LOADS]++;
      const f3 start_pos = add3(ray_pos, scl3(fNearFar.x, ray_dir));
      const f3 start_q = scl3(scale, sub3(start_pos, min_pos));
      const float qFar = (fNearFar.y - fNearFar.x) * scale;
      local_surface(c, type, ray_dir, instId, geomId, values, primId, d, 0.0f, qFar, fNearFar, start_q, hit);
      const uint32_t layout = h.aux_data & LRT_SBS_LAYOUT_MASK;
      if (c->rec && hit->t < old_t &&
          (layout == LRT_SBS_LAYOUT_ID32F_IRGB32F || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN)) {
        const uint32_t vx = (uint32_t)voxelPos.x, vy = (uint32_t)voxelPos.y, vz = (uint32_t)voxelPos.z;
        for (int i = 0; i < 8; i++) {
          const uint32_t vId = ((vx + ((i & 4) >> 2) + h.brick_pad) * v_size + (vy + ((i & 2) >> 1) + h.brick_pad)) *
                                   v_size + (vz + (i & 1) + h.brick_pad);
          c->rec->idx[i] = A->sdfSBSData[n->data_offset + vId];
        }
        c->rec->sbs = 1;
      }
    }
    bnf.x += smax(0.0f, fNearFar.y - bnf.x) + 1e-6f;
  }
  if (hit->t < old_t) {
    const uint32_t layout = h.aux_data & LRT_SBS_LAYOUT_MASK;
    if (layout == LRT_SBS_LAYOUT_ID32F_IRGB32F || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN) {
      /* colour of the hit (BVH2Common.cpp:1081-1110) */
      const f3 pos = add3(ray_pos, scl3(hit->t, ray_dir));
      const f3 dp = scl3(0.5f * sz, sub3(pos, brick_min_pos));
      const uint32_t t_off = n->data_offset + v_size * v_size * v_size;
      f3 col = mk3(0, 0, 0);
      for (int k = 0; k < 8; k++) {
        const uint32_t b = A->sdfSBSData[t_off + k];
        const float wx = (k & 4) ? dp.x : (1 - dp.x);
        const float wy = (k & 2) ? dp.y : (1 - dp.y);
        const float wz = (k & 1) ? dp.z : (1 - dp.z);
        const float w = wx * wy * wz;
        const f3 cc = scl3(w, mk3(A->sdfSBSDataF[b + 0], A->sdfSBSDataF[b + 1], A->sdfSBSDataF[b + 2]));
        col = (k == 0) ? cc : add3(col, cc);
      }
      col = mk3(sclamp(floorf(255.0f * col.x + 0.5f), 0.0f, 255.0f), sclamp(floorf(255.0f * col.y + 0.5f), 0.0f, 255.0f),
                sclamp(floorf(255.0f * col.z + 0.5f), 0.0f, 255.0f));
      hit->coords[0] = col.x + col.y / 256.0f;
      hit->coords[1] = col.z;
    }
  }
}

/* IntersectAllTrianglesInLeaf, BVH2Common.cpp:1571-1635 (NORMAL_MODE_GEOMETRY). */
static void triangles(ctx_t* c, f3 ray_pos, f3 ray_dir, float tNear, uint32_t instId, uint32_t geomId,
                      uint32_t a_start, uint32_t a_count, lrt_hit* hit)
{
  const lrt_scene_arrays* A = c->a;
  const uint32_t* go = A->geomData[geomId].offset;
  for (uint32_t triId = a_start; triId < a_start + a_count; triId++) {
    c->cnt[C_TRI_TESTS]++;
    const uint32_t ia = A->indices[go[0] + triId * 3 + 0];
    const uint32_t ib = A->indices[go[0] + triId * 3 + 1];
    const uint32_t ic = A->indices[go[0] + triId * 3 + 2];
    const f3 Ap = ld3(A->vertPos + 4 * (uint64_t)(go[1] + ia));
    const f3 Bp = ld3(A->vertPos + 4 * (uint64_t)(go[1] + ib));
    const f3 Cp = ld3(A->vertPos + 4 * (uint64_t)(go[1] + ic));
    const f3 edge1 = sub3(Bp, Ap);
    const f3 edge2 = sub3(Cp, Ap);
    const f3 pvec = cross3(ray_dir, edge2);
    const f3 tvec = sub3(ray_pos, Ap);
    const f3 qvec = cross3(tvec, edge1);
    const float invDet = 1.0f / dot3(edge1, pvec);
    const float v = dot3(tvec, pvec) * invDet;
    const float u = dot3(qvec, ray_dir) * invDet;
    const float t = dot3(edge2, qvec) * invDet;
    if (v >= -1e-6f && u >= -1e-6f && (u + v <= 1.0f + 1e-6f) && t > tNear && t < hit->t) {
      hit->t = t;
      hit->primId = triId;
      hit->instId = instId;
      hit->geomId = geomId | (LRT_TYPE_MESH_TRIANGLE << 24);
      hit->coords[0] = u;
      hit->coords[1] = v;
      if (need_normal(c->p)) {
        f3 nn = cross3(edge1, edge2);
        nn = normalize3(matmul4(A->instanceData[instId].transformInvTransposed, nn, 1.0f));
        const f2 en = encode_normal(nn);
        hit->coords[2] = en.x;
        hit->coords[3] = en.y;
      } else {
        hit->coords[2] = 0;
        hit->coords[3] = 0;
      }
    }
  }
}

/* IntersectAllPrimitivesInLeaf, BVH2Common.cpp:47-124 */
static uint32_t leaf(ctx_t* c, f3 ray_pos, f3 ray_dir, float tNear, uint32_t aabbId, uint32_t instId,
                     uint32_t geomId, lrt_hit* hit)
{
  const lrt_scene_arrays* A = c->a;
  const float tPrev = hit->t;
  c->cnt[C_LEAF_CALLS]++;
  const uint32_t globalAABBId = A->startEnd[2 * geomId] + aabbId;
  const uint32_t packed = A->primIdCount[globalAABBId];
  const uint32_t a_start = packed & START_MASK;
  const uint32_t a_count = (packed & SIZE_MASK) >> 28;
  const uint32_t tag = A->geomTags[geomId];
  switch (tag) {
    case LRT_TAG_TRIANGLE: triangles(c, ray_pos, ray_dir, tNear, instId, geomId, a_start, a_count, hit); break;
    case LRT_TAG_SDF_NODE:
      octree_node(c, A->geomData[geomId].type, ray_pos, ray_dir, tNear, instId, geomId, a_start, hit);
      break;
    case LRT_TAG_SDF_BRICK:
      octree_brick(c, A->geomData[geomId].type, ray_pos, ray_dir, tNear, instId, geomId, a_start, hit);
      break;
    default: break;
  }
  return (hit->t >= tPrev) ? LRT_TAG_NONE : tag;
}

/* BVHRT::BVH2TraverseF32, BVH2Common.cpp:3239-3320 */
static void blas(ctx_t* c, f3 ray_pos, f3 ray_dir, float tNear, uint32_t instId, uint32_t geomId, int stopOnFirstHit,
                 lrt_hit* hit)
{
  const lrt_scene_arrays* A = c->a;
  const uint32_t bvhOffset = A->geomData[geomId].bvhOffset;
  uint32_t stack[STACK_SIZE];
  int top = 0;
  uint32_t leftNodeOffset = 0;
  int hitFound = 0;
  stack[0] = 0;
  const f3 inv = safe_inverse(ray_dir);
  while (top >= 0 && !hitFound) {
    while (top >= 0 && ((leftNodeOffset & LEAF_BIT) == 0)) {
      c->cnt[C_BLAS_PAIRS]++;
      const lrt_bvh_node_pair* fat = &A->allNodePairs[bvhOffset + leftNodeOffset];
      const uint32_t n0 = fat->left.leftOffset, n1 = fat->right.leftOffset;
      const f2 tm0 = ray_box(ray_pos, inv, ld3(fat->left.boxMin), ld3(fat->left.boxMax));
      const f2 tm1 = ray_box(ray_pos, inv, ld3(fat->right.boxMin), ld3(fat->right.boxMax));
      const int h0 = (tm0.x <= tm0.y) && (tm0.y >= tNear) && (tm0.x <= hit->t);
      const int h1 = (tm1.x <= tm1.y) && (tm1.y >= tNear) && (tm1.x <= hit->t);
      leftNodeOffset = h0 ? n0 : n1;
      if (h0 && h1) {
        if (top >= STACK_SIZE) { c->limits++; return; }
        leftNodeOffset = (tm0.x <= tm1.x) ? n0 : n1;
        stack[top] = (tm0.x <= tm1.x) ? n1 : n0;
        top++;
      }
      if (!h0 && !h1) {
        top--;
        leftNodeOffset = stack[top > 0 ? top : 0];
      }
    }
    if (top >= 0 && leftNodeOffset != 0xFFFFFFFFu) {
      const float tNearSdf = smax(tNear, 0.01f); /* SDF_BIAS, :3306-3307 */
      const uint32_t tag = leaf(c, ray_pos, ray_dir, tNearSdf, leftNodeOffset & START_MASK, instId, geomId, hit);
      hitFound = (tag != 0) && (tag != LRT_TAG_TRIANGLE || stopOnFirstHit);
    }
    top--;
    leftNodeOffset = stack[top > 0 ? top : 0];
  }
}

/* BVHRT::RayQuery_NearestHit, BVH2Common.cpp:3322-3392 */
static lrt_hit nearest_hit(ctx_t* c, const float pn[4], const float dfar[4])
{
  const lrt_scene_arrays* A = c->a;
  float dirW = dfar[3];
  const int stopOnFirstHit = (dirW <= 0.0f);
  if (stopOnFirstHit) dirW *= -1.0f;
  const f3 pos = ld3(pn), dir = ld3(dfar);
  const float tmin = pn[3];
  const f3 inv = safe_inverse(dir);
  lrt_hit hit;
  hit.t = dirW;
  hit.primId = 0xFFFFFFFFu;
  hit.instId = 0xFFFFFFFFu;
  hit.geomId = 0xFFFFFFFFu;
  hit.coords[0] = 1.0f;
  hit.coords[1] = 0.0f;
  hit.coords[2] = 0.0f;
  hit.coords[3] = 0.0f;
  uint32_t nodeIdx = 0;
  uint64_t guard = 0;
  const uint64_t guard_max = 2 * A->nodesTLAS_count + 4;
  do {
    uint32_t travFlags = 0, leftOffset = 0;
    do {
      if (nodeIdx >= A->nodesTLAS_count || ++guard > guard_max) { c->limits++; goto done; }
      c->cnt[C_TLAS_NODES]++;
      const lrt_bvh_node* nd = &A->nodesTLAS[nodeIdx];
      const f2 bh = ray_box(pos, inv, ld3(nd->boxMin), ld3(nd->boxMax));
      const uint32_t intersects = (bh.x <= bh.y) && (bh.y > tmin) && (bh.x < hit.t);
      travFlags = (nd->leftOffset & LEAF_BIT) | intersects;
      leftOffset = nd->leftOffset;
      const int leafOrNot = (travFlags & LEAF_BIT) != 0 || (travFlags & 1) == 0;
      nodeIdx = leafOrNot ? nd->escapeIndex : leftOffset;
    } while (travFlags != (LEAF_BIT | 1u) && nodeIdx != 0 && nodeIdx < 0xFFFFFFFEu);
    if (travFlags == (LEAF_BIT | 1u)) {
      const uint32_t instId = leftOffset & START_MASK;
      const lrt_instance_data* inst = &A->instanceData[instId];
      const uint32_t geomId = inst->geomId;
      c->cnt[C_INSTANCES]++;
      const f3 rp = matmul4(inst->transformInv, pos, 1.0f);
      const f3 rd = matmul4(inst->transformInv, dir, 0.0f);
      blas(c, rp, rd, tmin, instId, geomId, stopOnFirstHit, &hit);
    }
  } while (nodeIdx < 0xFFFFFFFEu && !(stopOnFirstHit && hit.primId != 0xFFFFFFFFu));
done:
  if (hit.geomId < 0xFFFFFFFFu && ((hit.geomId >> 24) == LRT_TYPE_MESH_TRIANGLE)) {
    const uint32_t g = hit.geomId & 0x00FFFFFFu;
    c->tri_local = hit.primId;
    hit.primId = A->primIndices[A->geomData[g].offset[0] / 3 + hit.primId];
  }
  if (hit.primId != 0xFFFFFFFFu) c->cnt[C_HITS]++;
  return hit;
}

/* Trace n rays (n x {posAndNear, dirAndFar}).  counters may be NULL; it
 * receives LRT_COUNTER_COUNT sums.  Returns the number of bounded-loop /
 * bounds events (0 on well-formed scenes). */
uint64_t lrto_trace(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays, lrt_hit* hits,
                    uint64_t n, uint64_t* counters, int threads)
{
  uint64_t total[LRT_COUNTER_COUNT];
  memset(total, 0, sizeof(total));
  uint64_t limits = 0;
  (void)threads;
#ifdef _OPENMP
#pragma omp parallel num_threads(threads > 0 ? threads : 1) reduction(+ : limits)
#endif
  {
    uint64_t local[LRT_COUNTER_COUNT];
    memset(local, 0, sizeof(local));
    ctx_t c = {arrays, preset, local, 0};
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) hits[i] = nearest_hit(&c, rays + 8 * i, rays + 8 * i + 4);
    limits += c.limits;
#ifdef _OPENMP
#pragma omp critical
#endif
    for (int k = 0; k < LRT_COUNTER_COUNT; k++) total[k] += local[k];
  }
  if (counters)
    for (int k = 0; k < LRT_COUNTER_COUNT; k++) counters[k] = total[k];
  return limits;
}

/* Per-ray work counters (n x LRT_COUNTER_COUNT), single-threaded. */
void lrto_trace_counted(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays, lrt_hit* hits,
                        uint64_t n, uint64_t* per_ray_counters)
{
  for (uint64_t i = 0; i < n; i++) {
    ctx_t c = {arrays, preset, per_ray_counters + i * LRT_COUNTER_COUNT, 0};
    memset(c.cnt, 0, sizeof(uint64_t) * LRT_COUNTER_COUNT);
    hits[i] = nearest_hit(&c, rays + 8 * i, rays + 8 * i + 4);
  }
}

/* ------------------------------------------------------------------------ */
/* Lambert render and its FP64 adjoint (project-written; the reference has  */
/* no differentiable renderer).                                             */
/* ------------------------------------------------------------------------ */

/* decode_normal, utils/raytracing/render_common.h:257-266 */
static f3 decode_normal(float ex, float ey)
{
  f3 v = mk3(ex, ey, 1.0f - fabsf(ex) - fabsf(ey));
  if (v.z < 0) {
    const float vx = v.x;
    v.x = (1.0f - fabsf(v.y)) * ((v.x >= 0.0f) ? +1.0f : -1.0f);
    v.y = (1.0f - fabsf(vx)) * ((v.y >= 0.0f) ? +1.0f : -1.0f);
  }
  return normalize3(v);
}

/* ResolveCommon for LAMBERT_NO_TEX, one directional light of unit colour,
 * albedo 1 (MultiRenderer_resolve.cpp:617-666); triangle normals turned to
 * face the viewer as loadNormalTcFromGbuffer does (:58-59). */
static float lambert(const lrt_hit* h, f3 dir, f3 L)
{
  if (h->primId == 0xFFFFFFFFu) return 0.0f;
  f3 n = decode_normal(h->coords[2], h->coords[3]);
  if ((h->geomId >> 24) == LRT_TYPE_MESH_TRIANGLE) n = scl3(ssign(dot3(scl3(-1.0f, dir), n)), n);
  return smax(0.0f, dot3(n, L));
}

void lrto_render_lambert(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays, uint64_t n,
                         const float light[3], float* image, int threads)
{
  (void)threads;
  const f3 L = mk3(light[0], light[1], light[2]);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads > 0 ? threads : 1)
#endif
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t cnt[LRT_COUNTER_COUNT];
    ctx_t c = {arrays, preset, cnt, 0, NULL};
    const lrt_hit h = nearest_hit(&c, rays + 8 * i, rays + 8 * i + 4);
    image[i] = lambert(&h, ld3(rays + 8 * i + 4), L);
  }
}

/* FP64 reference adjoint: for every ray with dimage[i] != 0 whose nearest hit
 * lies on an indexed SBS brick, grad[idx_k] += dimage[i] * dI/dvalue_k with
 * the implicit-differentiation formula of the GPU kernel evaluated in double
 * (hit point, values and direction from the float march). */
void lrto_adjoint_lambert_fp64(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays,
                               uint64_t n, const float light[3], const float* dimage, double* grad)
{
  const f3 Lf = mk3(light[0], light[1], light[2]);
  const double L[3] = {light[0], light[1], light[2]};
  for (uint64_t i = 0; i < n; i++) {
    if (dimage[i] == 0.0f) continue;
    uint64_t cnt[LRT_COUNTER_COUNT];
    hit_record_t rec;
    rec.t = -1.0f;
    rec.sbs = 0;
    ctx_t c = {arrays, preset, cnt, 0, &rec};
    const lrt_hit h = nearest_hit(&c, rays + 8 * i, rays + 8 * i + 4);
    if (h.primId == 0xFFFFFFFFu || !rec.sbs || rec.t != h.t) continue;
    if (lambert(&h, ld3(rays + 8 * i + 4), Lf) <= 0.0f) continue;
    const float* Mf = arrays->instanceData[h.instId].transformInvTransposed;
    double M[16];
    for (int k = 0; k < 16; k++) M[k] = Mf[k];
    const double p[3] = {rec.p.x, rec.p.y, rec.p.z}, dir[3] = {rec.dir.x, rec.dir.y, rec.dir.z};
    double g[3] = {0, 0, 0}, hxy = 0, hxz = 0, hyz = 0, w[8], dw[8][3];
    for (int k = 0; k < 8; k++) {
      const double sx = (k & 4) ? 1 : -1, sy = (k & 2) ? 1 : -1, sz = (k & 1) ? 1 : -1;
      const double wx = (k & 4) ? p[0] : 1 - p[0], wy = (k & 2) ? p[1] : 1 - p[1], wz = (k & 1) ? p[2] : 1 - p[2];
      const double v = rec.values[k];
      w[k] = wx * wy * wz;
      dw[k][0] = sx * wy * wz;
      dw[k][1] = wx * sy * wz;
      dw[k][2] = wx * wy * sz;
      for (int a = 0; a < 3; a++) g[a] += v * dw[k][a];
      hxy += v * sx * sy * wz;
      hxz += v * sx * wy * sz;
      hyz += v * wx * sy * sz;
    }
    double m[3];
    for (int r = 0; r < 3; r++) m[r] = M[r] * g[0] + M[4 + r] * g[1] + M[8 + r] * g[2];
    const double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
    const double nn[3] = {m[0] / len, m[1] / len, m[2] / len};
    const double nl = nn[0] * L[0] + nn[1] * L[1] + nn[2] * L[2];
    const double q[3] = {(L[0] - nl * nn[0]) / len, (L[1] - nl * nn[1]) / len, (L[2] - nl * nn[2]) / len};
    const double u[3] = {M[0] * q[0] + M[1] * q[1] + M[2] * q[2], M[4] * q[0] + M[5] * q[1] + M[6] * q[2],
                         M[8] * q[0] + M[9] * q[1] + M[10] * q[2]};
    const double Hd[3] = {hxy * dir[1] + hxz * dir[2], hxy * dir[0] + hyz * dir[2], hxz * dir[0] + hyz * dir[1]};
    const double uHd = u[0] * Hd[0] + u[1] * Hd[1] + u[2] * Hd[2];
    const double gd = g[0] * dir[0] + g[1] * dir[1] + g[2] * dir[2];
    if (gd == 0.0 && !rec.early) continue;
    for (int k = 0; k < 8; k++) {
      const double dn = u[0] * dw[k][0] + u[1] * dw[k][1] + u[2] * dw[k][2];
      const double dI = rec.early ? dn : dn - uHd * w[k] / gd; /* early hits: the hit point is fixed */
      grad[rec.idx[k]] += (double)dimage[i] * dI;
    }
  }
}

/* Lambert intensity of the FP64 surface model of one hit voxel: the root of
 * the trilinear field along the ray next to the recorded hit point (Newton),
 * or the recorded point itself for an early hit (the voxel entry point the
 * march stopped at), its normal M grad f / |M grad f| and max(0, n . L). */
static double model_intensity(const double v[8], const double p0[3], const double dir[3], const double M[16],
                              const double L[3], int early)
{
  double s = 0.0, p[3] = {p0[0], p0[1], p0[2]}, g[3];
  for (int it = 0; it < (early ? 1 : 50); it++) {
    p[0] = p0[0] + s * dir[0];
    p[1] = p0[1] + s * dir[1];
    p[2] = p0[2] + s * dir[2];
    double f = 0;
    g[0] = g[1] = g[2] = 0;
    for (int k = 0; k < 8; k++) {
      const double wx = (k & 4) ? p[0] : 1 - p[0], wy = (k & 2) ? p[1] : 1 - p[1], wz = (k & 1) ? p[2] : 1 - p[2];
      const double sx = (k & 4) ? 1 : -1, sy = (k & 2) ? 1 : -1, sz = (k & 1) ? 1 : -1;
      f += v[k] * wx * wy * wz;
      g[0] += v[k] * sx * wy * wz;
      g[1] += v[k] * wx * sy * wz;
      g[2] += v[k] * wx * wy * sz;
    }
    const double df = g[0] * dir[0] + g[1] * dir[1] + g[2] * dir[2];
    if (df == 0.0) break;
    const double step = f / df;
    s -= step;
    if (fabs(step) < 1e-15) break;
  }
  double m[3];
  for (int r = 0; r < 3; r++) m[r] = M[r] * g[0] + M[4 + r] * g[1] + M[8 + r] * g[2];
  const double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  const double nl = (m[0] * L[0] + m[1] * L[1] + m[2] * L[2]) / len;
  return nl > 0 ? nl : 0.0;
}

/* |cos| of the angle between the ray and the model's field gradient at the
 * unperturbed hit, and n . L there (the quantities whose small values make
 * the intensity a steep or kinked function of the voxel values: grazing rays,
 * where dt/dtheta ~ 1/(grad f . d), and the max(0, n . L) terminator). */
static void model_shape(const double v[8], const double p0[3], const double dir[3], const double M[16],
                        const double L[3], int early, double* cosgd, double* nl_out)
{
  double s = 0.0, p[3], g[3] = {0, 0, 0};
  for (int it = 0; it < (early ? 1 : 50); it++) {
    for (int r = 0; r < 3; r++) p[r] = p0[r] + s * dir[r];
    double f = 0;
    g[0] = g[1] = g[2] = 0;
    for (int k = 0; k < 8; k++) {
      const double wx = (k & 4) ? p[0] : 1 - p[0], wy = (k & 2) ? p[1] : 1 - p[1], wz = (k & 1) ? p[2] : 1 - p[2];
      const double sx = (k & 4) ? 1 : -1, sy = (k & 2) ? 1 : -1, sz = (k & 1) ? 1 : -1;
      f += v[k] * wx * wy * wz;
      g[0] += v[k] * sx * wy * wz;
      g[1] += v[k] * wx * sy * wz;
      g[2] += v[k] * wx * wy * sz;
    }
    const double df = g[0] * dir[0] + g[1] * dir[1] + g[2] * dir[2];
    if (df == 0.0) break;
    const double step = f / df;
    s -= step;
    if (fabs(step) < 1e-15) break;
  }
  const double gl = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  const double dl = sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
  const double gd = g[0] * dir[0] + g[1] * dir[1] + g[2] * dir[2];
  *cosgd = (gl > 0 && dl > 0) ? fabs(gd) / (gl * dl) : 0.0;
  double m[3];
  for (int r = 0; r < 3; r++) m[r] = M[r] * g[0] + M[4 + r] * g[1] + M[8 + r] * g[2];
  const double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  *nl_out = len > 0 ? (m[0] * L[0] + m[1] * L[1] + m[2] * L[2]) / len : 0.0;
}

/* Central differences (step h, in double) of sum_i dimage[i] * I_i with
 * respect to the value indices `keys` (sorted ascending), where I_i is the
 * FP64 surface model of ray i's hit voxel.  This checks the implicit-
 * differentiation formula without the rounding noise of the float32 march.
 * Where min_cos / min_nl are not NULL they receive, per key, the smallest
 * |cos(grad f, d)| and n . L over the pixels whose hit voxel has that value
 * as a corner (1 and +inf for keys no pixel reaches). */
void lrto_fd_model_fp64_shape(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays,
                              uint64_t n, const float light[3], const float* dimage, const uint32_t* keys,
                              uint64_t nkeys, double h, double* out, double* min_cos, double* min_nl, int threads);

void lrto_fd_model_fp64(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays, uint64_t n,
                        const float light[3], const float* dimage, const uint32_t* keys, uint64_t nkeys, double h,
                        double* out, int threads)
{
  lrto_fd_model_fp64_shape(arrays, preset, rays, n, light, dimage, keys, nkeys, h, out, NULL, NULL, threads);
}

void lrto_fd_model_fp64_shape(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays,
                              uint64_t n, const float light[3], const float* dimage, const uint32_t* keys,
                              uint64_t nkeys, double h, double* out, double* min_cos, double* min_nl, int threads)
{
  if (min_cos)
    for (uint64_t k = 0; k < nkeys; k++) min_cos[k] = 1.0;
  if (min_nl)
    for (uint64_t k = 0; k < nkeys; k++) min_nl[k] = INFINITY;
  const f3 Lf = mk3(light[0], light[1], light[2]);
  const double L[3] = {light[0], light[1], light[2]};
  (void)threads;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1024) num_threads(threads > 0 ? threads : 1)
#endif
  for (int64_t i = 0; i < (int64_t)n; i++) {
    if (dimage[i] == 0.0f) continue;
    uint64_t cnt[LRT_COUNTER_COUNT];
    hit_record_t rec;
    rec.t = -1.0f;
    rec.sbs = 0;
    ctx_t c = {arrays, preset, cnt, 0, &rec};
    const lrt_hit hh = nearest_hit(&c, rays + 8 * i, rays + 8 * i + 4);
    if (hh.primId == 0xFFFFFFFFu || !rec.sbs || rec.t != hh.t) continue;
    if (lambert(&hh, ld3(rays + 8 * i + 4), Lf) <= 0.0f) continue;
    const float* Mf = arrays->instanceData[hh.instId].transformInvTransposed;
    double M[16], v[8];
    for (int k = 0; k < 16; k++) M[k] = Mf[k];
    for (int k = 0; k < 8; k++) v[k] = rec.values[k];
    const double p0[3] = {rec.p.x, rec.p.y, rec.p.z}, dir[3] = {rec.dir.x, rec.dir.y, rec.dir.z};
    for (int k = 0; k < 8; k++) {
      uint64_t lo = 0, hi = nkeys;
      while (lo < hi) {
        const uint64_t mid = (lo + hi) / 2;
        if (keys[mid] < rec.idx[k]) lo = mid + 1; else hi = mid;
      }
      if (lo >= nkeys || keys[lo] != rec.idx[k]) continue;
      double vp[8], vm[8];
      for (int j = 0; j < 8; j++) vp[j] = vm[j] = v[j];
      vp[k] += h;
      vm[k] -= h;
      const double d =
          (model_intensity(vp, p0, dir, M, L, rec.early) - model_intensity(vm, p0, dir, M, L, rec.early)) / (2 * h);
#ifdef _OPENMP
#pragma omp atomic
#endif
      out[lo] += (double)dimage[i] * d;
      if (min_cos || min_nl) {
        double cg, nl;
        model_shape(v, p0, dir, M, L, rec.early, &cg, &nl);
#ifdef _OPENMP
#pragma omp critical(lrto_fd_shape)
#endif
        {
          if (min_cos && cg < min_cos[lo]) min_cos[lo] = cg;
          if (min_nl && nl < min_nl[lo]) min_nl[lo] = nl;
        }
      }
    }
  }
}


/* ------------------------------------------------------------------------ */
/* MultiRenderer::Render for LAMBERT_NO_TEX, one sample, no transparency    */
/* (MultiRenderer.cpp:14-60): ResolveCommon + Tonemap of each eye ray.      */
/* ------------------------------------------------------------------------ */

/* Tonemap, MultiRenderer_resolve.cpp:536-542: uint4(255 * clamp(c, 0, 1)). */
static uint32_t tonemap_rgba8(float r, float g, float b, float a)
{
  const uint32_t x = (uint32_t)(255.0f * sclamp(r, 0.0f, 1.0f));
  const uint32_t y = (uint32_t)(255.0f * sclamp(g, 0.0f, 1.0f));
  const uint32_t z = (uint32_t)(255.0f * sclamp(b, 0.0f, 1.0f));
  const uint32_t w = (uint32_t)(255.0f * sclamp(a, 0.0f, 1.0f));
  return (w << 24) | (z << 16) | (y << 8) | x;
}

/* rays: the eye rays of the image in row-major pixel order (initEyeRay). */
/* MultiRenderer's palettes (MultiRenderer.h:269-283) and decode_RGBA8
 * (utils/raytracing/render_common.h:250-254). */
static const uint32_t kPalette[20] = {0xffe6194b, 0xff3cb44b, 0xffffe119, 0xff0082c8, 0xfff58231,
                                      0xff911eb4, 0xff46f0f0, 0xfff032e6, 0xffd2f53c, 0xfffabebe,
                                      0xff008080, 0xffe6beff, 0xffaa6e28, 0xfffffac8, 0xff800000,
                                      0xffaaffc3, 0xff808000, 0xffffd8b1, 0xff000080, 0xff808080};
static const uint32_t kLodPalette[20] = {0xff000000, 0xff000040, 0xff000080, 0xff0000c0, 0xff0040ff,
                                         0xff0080ff, 0xff00c0ff, 0xff00ffff, 0xff00ffc0, 0xff00ff80,
                                         0xff00ff40, 0xff00ff00, 0xff00c000, 0xff008000, 0xff004000,
                                         0xff000000, 0xffff0000, 0xffff0000, 0xffff0000, 0xffff0000};
static void decode_rgba8(uint32_t c, float out[4])
{
  out[0] = (float)(c & 0xFF) * (1.0f / 255.0f);
  out[1] = (float)((c >> 8) & 0xFF) * (1.0f / 255.0f);
  out[2] = (float)((c >> 16) & 0xFF) * (1.0f / 255.0f);
  out[3] = (float)((c >> 24) & 0xFF) * (1.0f / 255.0f);
}

/* The renderer's textures and the meshes' texture coordinates for the
 * resolve (MultiRenderer::m_textures, MultiRenderer.h:256; the per-vertex
 * coordinates add_mesh_internal keeps in m_vertices[].w / m_normals[].w,
 * MultiRenderer_host.cpp:499-520).  Texture k: dims[2k] x dims[2k+1] float4
 * texels, row-major, from texel offset tex_off[k] of texels; vert_tc: two
 * floats per vertex of the scene's vertex array (NULL: all zero).  Set with
 * lrto_set_textures before a render call (test infrastructure: one set per
 * process, not thread-safe). */
static struct {
  const float* texels;
  const uint32_t* dims;
  const uint64_t* tex_off;
  uint32_t count;
  const float* vert_tc;
  uint64_t nverts;
} g_tex;

void lrto_set_textures(const float* texels, const uint32_t* dims, const uint64_t* tex_off, uint32_t count,
                       const float* vert_tc, uint64_t nverts)
{
  g_tex.texels = texels;
  g_tex.dims = dims;
  g_tex.tex_off = tex_off;
  g_tex.count = count;
  g_tex.vert_tc = vert_tc;
  g_tex.nverts = nverts;
}

/* Image2D<float4>::sample (dependencies/1st-party/LiteMath/Image2d.cpp:105-183)
 * with the sampler every MultiRenderer texture has (AddTexture,
 * MultiRenderer_host.cpp:827-839): LINEAR filter, CLAMP in both directions
 * (bilinearOffsets, Image2d.cpp:50-102). */
static void sample_texture(uint32_t tex, float u, float v, float out[4])
{
  if (tex >= g_tex.count) { out[0] = out[1] = out[2] = out[3] = 0.0f; return; }
  const int w = (int)g_tex.dims[2 * tex], hgt = (int)g_tex.dims[2 * tex + 1];
  const float* data = g_tex.texels + 4 * g_tex.tex_off[tex];
  float ffx = u * (float)w - 0.5f;
  float ffy = v * (float)hgt - 0.5f;
  if (ffx < 0) ffx = 0.0f;
  if (ffy < 0) ffy = 0.0f;
  const int px = (int)ffx, py = (int)ffy;
  const float fx = fabsf(ffx - (float)px), fy = fabsf(ffy - (float)py);
  const float fx1 = 1.0f - fx, fy1 = 1.0f - fy;
  const float w1 = fx1 * fy1, w2 = fx * fy1, w3 = fx1 * fy, w4 = fx * fy;
  int px0 = px >= w ? w - 1 : px, px1 = px + 1 >= w ? w - 1 : px + 1;
  int py0 = py >= hgt ? hgt - 1 : py, py1 = py + 1 >= hgt ? hgt - 1 : py + 1;
  px0 = px0 < 0 ? 0 : px0;
  px1 = px1 < 0 ? 0 : px1;
  py0 = py0 < 0 ? 0 : py0;
  py1 = py1 < 0 ? 0 : py1;
  const float* f1 = data + 4 * ((int64_t)py0 * w + px0);
  const float* f2 = data + 4 * ((int64_t)py0 * w + px1);
  const float* f3 = data + 4 * ((int64_t)py1 * w + px0);
  const float* f4 = data + 4 * ((int64_t)py1 * w + px1);
  for (int k = 0; k < 4; k++) out[k] = f1[k] * w1 + f2[k] * w2 + f3[k] * w3 + f4[k] * w4;
}

/* ResolveCommon (MultiRenderer_resolve.cpp:580-666) / kernel1D_ResolveDebug
 * (:810-990) of hit h for `mode`, with the resolve ray r (initEyeRay of
 * sample 0) and c->tri_local of the trace that found h: the float4 colour
 * before Tonemap (alpha 1 for hits, the background's for misses).  Modes:
 * MASK, LAMBERT_NO_TEX, DEPTH, LINEAR_DEPTH, INVERSE_LINEAR_DEPTH, PRIMITIVE,
 * TYPE, GEOM, NORMAL, BARYCENTRIC, ST_ITERATIONS, PHONG_NO_TEX, DIFFUSE,
 * LAMBERT, PHONG, HSV_DEPTH, LOD, MATERIAL, MO_VOXEL_COUNT, MO_FLAGS;
 * materials COLORED only (offsets {start, size} per geometry; may be NULL
 * for the modes that read none). */
static void resolve_colour(const lrt_scene_arrays* arrays, const ctx_t* cp, uint32_t mode, lrt_hit h, const float* r,
                           const lrt_light* lights, uint32_t light_count, const float background[4],
                           const lrt_material* materials, const uint32_t* mat_ids, const uint32_t* mat_offsets,
                           float out[4])
{
  const ctx_t cc = *cp;
  const ctx_t* c = &cc;
  if (h.primId == 0xFFFFFFFFu) {
    memcpy(out, background, 4 * sizeof(float));
    return;
  }
  {
    const uint32_t type = h.geomId >> 24, geomId = h.geomId & 0x00FFFFFFu;
    const f3 rayPos = mk3(r[0], r[1], r[2]), rayDir = mk3(r[4], r[5], r[6]);
    f3 norm;
    float tcu = h.coords[0], tcv = h.coords[1]; /* loadNormalTcFromGbuffer's tc (:27-76) */
    if (type == LRT_TYPE_MESH_TRIANGLE) {
      /* loadNormalTcFromGbuffer, NORMAL_MODE_GEOMETRY (:33-59) */
      const uint32_t g = geomId;
      const uint32_t base = arrays->geomData[g].offset[0] + 3 * c->tri_local;
      float tcs[3][2] = {{0, 0}, {0, 0}, {0, 0}};
      for (int k = 0; k < 3; k++) {
        const uint64_t vi = (uint64_t)arrays->geomData[g].offset[1] + arrays->indices[base + k];
        if (g_tex.vert_tc && vi < g_tex.nverts) {
          tcs[k][0] = g_tex.vert_tc[2 * vi];
          tcs[k][1] = g_tex.vert_tc[2 * vi + 1];
        }
      }
      /* (1 - c0 - c1) * A_tc + c1 * B_tc + c0 * C_tc */
      const float wa = 1.0f - h.coords[0] - h.coords[1];
      tcu = wa * tcs[0][0] + h.coords[1] * tcs[1][0] + h.coords[0] * tcs[2][0];
      tcv = wa * tcs[0][1] + h.coords[1] * tcs[1][1] + h.coords[0] * tcs[2][1];
      const float* vA = arrays->vertPos + 4 * (uint64_t)(arrays->geomData[g].offset[1] + arrays->indices[base + 0]);
      const float* vB = arrays->vertPos + 4 * (uint64_t)(arrays->geomData[g].offset[1] + arrays->indices[base + 1]);
      const float* vC = arrays->vertPos + 4 * (uint64_t)(arrays->geomData[g].offset[1] + arrays->indices[base + 2]);
      const f3 A = mk3(vA[0], vA[1], vA[2]), B = mk3(vB[0], vB[1], vB[2]), C = mk3(vC[0], vC[1], vC[2]);
      const f3 raw = cross3(sub3(B, A), sub3(C, A));
      norm = normalize3(matmul4(arrays->instanceData[h.instId].transformInvTransposed, raw, 1.0f));
      norm = scl3(ssign(dot3(scl3(-1.0f, rayDir), norm)), norm);
    } else {
      norm = decode_normal(h.coords[2], h.coords[3]);
    }
    /* m_matIdbyPrimId[m_matIdOffsets[geomId].x + primId % m_matIdOffsets[geomId].y] */
#define MAT_ID() (mat_ids[mat_offsets[2 * geomId] + h.primId % mat_offsets[2 * geomId + 1]])
    /* a material's colour: base_color if COLORED, else its texture at tc */
    float mc[4];
#define MAT_COLOUR(m)                                                            \
  do {                                                                           \
    if ((m)->type == LRT_MATERIAL_COLORED) memcpy(mc, (m)->base_color, sizeof(mc)); \
    else sample_texture((m)->texId, tcu, tcv, mc);                                 \
  } while (0)
    const float z = h.t, z_near = 0.1f, z_far = 10.0f;
    float res[4] = {1, 0, 1, 1};
    switch (mode) {
    case 0: res[0] = res[1] = res[2] = res[3] = 1; break; /* MASK */
    case 2: { /* DEPTH */
      const float d = (1.0f / z - 1.0f / z_near) / (1.0f / z_far - 1.0f / z_near);
      res[0] = res[1] = res[2] = d;
    } break;
    case 3: { /* LINEAR_DEPTH */
      const float d = (z - z_near) / (z_far - z_near);
      res[0] = res[1] = res[2] = d;
    } break;
    case 4: { /* INVERSE_LINEAR_DEPTH */
      const float d = 1 - ((z - z_near) / (z_far - z_near));
      res[0] = res[1] = res[2] = d;
    } break;
    case 5: case 25: decode_rgba8(kPalette[h.primId % 20], res); break; /* PRIMITIVE, MO_FLAGS */
    case 6: decode_rgba8(kPalette[type % 20], res); break;               /* TYPE */
    case 22: decode_rgba8(kPalette[MAT_ID() % 20], res); break;          /* MATERIAL */
    case 8: { /* NORMAL */
      const float vx = fabsf(norm.x), vy = fabsf(norm.y), vz = fabsf(norm.z);
      res[0] = 0.25f + 0.5f * powf(vx, 1.0f / 1.5f);
      res[1] = 0.25f + 0.5f * powf(vy, 1.0f / 1.5f);
      res[2] = 0.25f + 0.5f * powf(vz, 1.0f / 1.5f);
    } break;
    case 9: /* BARYCENTRIC */
      res[0] = h.coords[0];
      res[1] = h.coords[1];
      res[2] = 1 - h.coords[0] - h.coords[1];
      break;
    case 10: /* ST_ITERATIONS */
      if (h.primId == 0) {
        res[0] = res[1] = res[2] = 0.5f;
      } else if (h.primId <= 64) {
        const float q = sclamp((float)h.primId / 64, 0.0f, 1.0f);
        res[0] = q * 0 + (1.0f - q) * 0;
        res[1] = q * 0 + (1.0f - q) * 1;
        res[2] = q * 1 + (1.0f - q) * 0;
      } else {
        const float q = sclamp((float)(h.primId - 64) / (256 - 64), 0.0f, 1.0f);
        res[0] = q * 1 + (1.0f - q) * 0;
        res[1] = q * 0 + (1.0f - q) * 0;
        res[2] = q * 0 + (1.0f - q) * 1;
      }
      break;
    case 24: /* MO_VOXEL_COUNT */
      if (h.primId == 0) { res[0] = 0.5f; res[1] = 0.5f; res[2] = 0.5f; }
      else if (h.primId == 1) { res[0] = 0.5f; res[1] = 1; res[2] = 0.5f; }
      else if (h.primId == 2) { res[0] = 0.5f; res[1] = 0.5f; res[2] = 1; }
      else if (h.primId <= 64) {
        const float q = sclamp((float)h.primId / 64, 0.0f, 1.0f);
        res[0] = q * 1 + (1 - q) * 0.5f;
        res[1] = q * 0 + (1 - q) * 0.5f;
        res[2] = q * 0 + (1 - q) * 1;
      } else { res[0] = 1; res[1] = 0; res[2] = 0; }
      break;
    case 19: { /* HSV_DEPTH */
      const f3 isect = add3(rayPos, scl3(z, rayDir));
      float zt = (isect.z + 1.f) * 2.f;
      zt = zt - (float)(int)zt;
      if (zt < 0.f) zt = 1.f + zt;
      const float hx = zt, hy = 1.f, hz = 1.f;
      float col[4] = {hz, hz, hz, 1.f};
      const float vmin = (1.f - hy) * hz;
      float Hi = 0.f;
      const float a = (hz - vmin) * modff(hx * 6.f, &Hi);
      uint32_t H = (uint32_t)Hi;
      H = H <= 5u ? H : 5u;
      col[(2u + (H >> 1)) % 3u] = vmin;
      if ((H & 1u) != 0u) col[H >> 1] = hz - a;
      else col[(1u + (H >> 1)) % 3u] = vmin + a;
      res[0] = col[0]; res[1] = col[1]; res[2] = col[2];
    } break;
    case 16: { /* DIFFUSE, COLORED materials */
      if (type == LRT_TYPE_SDF_SBS_COL) {
        res[0] = roundf(h.coords[0]) / 255.0f;
        res[1] = h.coords[0] - floorf(h.coords[0]);
        res[2] = roundf(h.coords[1]) / 255.0f;
      } else {
        const lrt_material* m = &materials[MAT_ID()];
        MAT_COLOUR(m);
        res[0] = mc[0]; res[1] = mc[1]; res[2] = mc[2];
      }
    } break;
    case 15: /* TEX_COORDS */
      res[0] = tcu;
      res[1] = tcv;
      res[2] = 0;
      break;
    case 1: case 7: case 13: case 17: case 20: { /* LAMBERT_NO_TEX, GEOM, OUTLINE_PRIM, LAMBERT (COLORED), LOD */
      f3 color = mk3(0, 0, 1);
      float pc[4];
      if (mode == 1 || mode == 13) color = mk3(1, 1, 1);
      else if (mode == 20) { decode_rgba8(kLodPalette[h.primId % 20], pc); color = mk3(pc[0], pc[1], pc[2]); }
      else if (mode == 7) { decode_rgba8(kPalette[geomId % 20], pc); color = mk3(pc[0], pc[1], pc[2]); }
      else if (type == LRT_TYPE_SDF_SBS_COL || type == LRT_TYPE_GRAPHICS_PRIM)
        color = mk3(roundf(h.coords[0]) / 255.0f, h.coords[0] - floorf(h.coords[0]), roundf(h.coords[1]) / 255.0f);
      else {
        const lrt_material* m = &materials[MAT_ID()];
        MAT_COLOUR(m);
        color = mk3(mc[0], mc[1], mc[2]);
      }
      f3 fc = mk3(0, 0, 0);
      for (uint32_t k = 0; k < light_count; k++) {
        const lrt_light* l = &lights[k];
        const f3 lc = mk3(l->color[0], l->color[1], l->color[2]);
        const f3 sp = mk3(l->space[0], l->space[1], l->space[2]);
        if (l->type == LRT_LIGHT_DIRECT) {
          const float q = smax(0.0f, dot3(norm, sp));
          fc = add3(fc, scl3(q, mul3(lc, color)));
        } else if (l->type == LRT_LIGHT_POINT) {
          const f3 surf = add3(rayPos, scl3(h.t, rayDir));
          f3 dir = sub3(sp, surf);
          const float len = sqrtf(dot3(dir, dir));
          dir = mk3(dir.x / len, dir.y / len, dir.z / len);
          const float q = smax(0.0f, dot3(norm, dir));
          const f3 lq = scl3(q, mul3(lc, color));
          fc = add3(fc, mk3(lq.x / (len * len), lq.y / (len * len), lq.z / (len * len)));
        } else {
          fc = add3(fc, mul3(lc, color));
        }
      }
      res[0] = fc.x; res[1] = fc.y; res[2] = fc.z;
    } break;
    case 11: case 21: { /* PBR_NO_TEX (material 0), PBR (COLORED) */
      const lrt_material* m = mode == 11 ? &materials[0] : &materials[MAT_ID()];
      MAT_COLOUR(m);
      const f3 baseColor = mk3(mc[0], mc[1], mc[2]);
      const float metallic = m->metallic, roughness = m->roughness;
      const float alpha = roughness * roughness, f0 = 0.04f;
      const f3 surf = add3(rayPos, scl3(h.t, rayDir));
      const f3 eye_dir = scl3(-1.0f, rayDir);
      const float NV = dot3(norm, eye_dir);
      f3 fc = mk3(0, 0, 0);
      for (uint32_t k = 0; k < light_count; k++) {
        const lrt_light* l = &lights[k];
        f3 light_dir = mk3(1, 1, 1);
        if (l->type == LRT_LIGHT_DIRECT) {
          light_dir = mk3(l->space[0], l->space[1], l->space[2]);
        } else if (l->type == LRT_LIGHT_POINT) {
          light_dir = sub3(mk3(l->space[0], l->space[1], l->space[2]), surf);
          const float len = sqrtf(dot3(light_dir, light_dir));
          light_dir = mk3(light_dir.x / len, light_dir.y / len, light_dir.z / len);
        }
        f3 half = add3(eye_dir, light_dir);
        const float hl = sqrtf(dot3(half, half));
        half = mk3(half.x / hl, half.y / hl, half.z / hl);
        const float NH = dot3(norm, half), NL = dot3(norm, light_dir), HL = dot3(half, light_dir),
                    HV = dot3(half, eye_dir);
        const float D = alpha * smax(0.0f, NH) / smax(LRT_PI_F * powf(NH * NH * (alpha - 1.0f) + 1.0f, 2.0f), 0.00001f);
        float V = smax(0.0f, HL) / smax(fabsf(NL) + sqrtf(alpha + (1 - alpha) * NL * NL), 0.00001f);
        V *= smax(0.0f, HV) / smax(fabsf(NV) + sqrtf(alpha + (1 - alpha) * NV * NV), 0.00001f);
        const float spec = V * D;
        const float ip = 1.0f / LRT_PI_F;
        const f3 diffuse = scl3(ip, baseColor);
        const float p5 = powf(1.0f - fabsf(HV), 5.0f);
        const f3 metal = scl3(spec, mk3(baseColor.x + (1.0f - baseColor.x) * p5, baseColor.y + (1.0f - baseColor.y) * p5,
                                        baseColor.z + (1.0f - baseColor.z) * p5));
        const float F = f0 + (1.0f - f0) * p5;
        const float fs = F * spec;
        const f3 diel = mk3((1.0f - F) * diffuse.x + fs, (1.0f - F) * diffuse.y + fs, (1.0f - F) * diffuse.z + fs);
        const f3 brdf = add3(scl3(1.0f - metallic, diel), scl3(metallic, metal));
        fc = add3(fc, scl3(smax(NL, 0.0f), brdf));
      }
      res[0] = fc.x; res[1] = fc.y; res[2] = fc.z;
    } break;
    case 12: case 18: { /* PHONG_NO_TEX, PHONG (COLORED); the shadow ray is commented out (shade = 1) */
      const float Kd = 0.25f, Ks = 0.25f, BIAS = 1e-6f;
      f3 color = mk3(0, 0, 1);
      if (mode == 12) color = mk3(1, 1, 1);
      else if (type == LRT_TYPE_SDF_SBS_COL || type == LRT_TYPE_GRAPHICS_PRIM)
        color = mk3(roundf(h.coords[0]) / 255.0f, h.coords[0] - floorf(h.coords[0]), roundf(h.coords[1]) / 255.0f);
      else {
        const lrt_material* m = &materials[MAT_ID()];
        MAT_COLOUR(m);
        color = mk3(mc[0], mc[1], mc[2]);
      }
      f3 fc = mk3(0, 0, 0);
      for (uint32_t k = 0; k < light_count; k++) {
        const lrt_light* l = &lights[k];
        const f3 lc = mk3(l->color[0], l->color[1], l->color[2]);
        const f3 sp = mk3(l->space[0], l->space[1], l->space[2]);
        if (l->type == LRT_LIGHT_AMBIENT) {
          fc = add3(fc, mul3(lc, color));
          continue;
        }
        const f3 surf = add3(rayPos, scl3(h.t - BIAS, rayDir));
        f3 light_dir = mk3(1, 1, 1);
        if (l->type == LRT_LIGHT_DIRECT) {
          light_dir = sp;
          const float q = smax(0.0f, dot3(norm, sp));
          fc = add3(fc, scl3(q, mul3(lc, color)));
        } else if (l->type == LRT_LIGHT_POINT) {
          const f3 dir = sub3(sp, surf);
          const float len = sqrtf(dot3(dir, dir));
          light_dir = mk3(dir.x / len, dir.y / len, dir.z / len);
        }
        const f3 refl = add3(scl3(-1.0f, light_dir), scl3(2.0f * dot3(norm, light_dir), norm));
        /* std::pow(float, int) is the double overload */
        const double spec = (double)Ks * pow((double)smax(0.0f, dot3(norm, refl)), 32);
        const float kk = (float)((double)(Kd * smax(0.0f, dot3(norm, light_dir))) + spec);
        fc = add3(fc, mul3(scl3(kk, scl3(1.0f, lc)), color));
      }
      res[0] = fc.x; res[1] = fc.y; res[2] = fc.z;
    } break;
    default: break;
    }
#undef MAT_ID
#undef MAT_COLOUR
    out[0] = res[0];
    out[1] = res[1];
    out[2] = res[2];
    out[3] = 1.0f;
  }
}


/* MultiRenderer::AnyHit (MultiRenderer.cpp:223-246) for the eye ray r:
 * nearest hits composited front to back, each trace restarting at the
 * previous hit point; offsets are {start, size} per geometry.  The loop is
 * the reference's, bounded by max_layers traces (the reference has no
 * bound); returns 1 if it reached that bound. */
static int anyhit(ctx_t* c, const float* r, const lrt_material* materials, const uint32_t* mat_ids,
                  const uint32_t* mat_offsets, const float background[4], uint32_t max_layers, lrt_hit* out,
                  f3* out_tc, float* out_alpha)
{
  float pn[4] = {r[0], r[1], r[2], r[3]};
  f3 tc = mk3(0, 0, 0);
  float alpha = 1.0f;
  float color[4] = {0, 0, 0, 0};
  lrt_hit h;
  uint32_t layer = 0;
  int capped = 0;
  memset(&h, 0, sizeof(h));
  do {
    if (layer++ == max_layers) {
      capped = 1;
      break;
    }
    /* transparencyColor += alpha * color.w * to_float3(color) */
    const float wa = alpha * color[3];
    tc = mk3(tc.x + wa * color[0], tc.y + wa * color[1], tc.z + wa * color[2]);
    alpha *= (1.0f - color[3]);
    h = nearest_hit(c, pn, r + 4);
    const uint32_t type = h.geomId >> 24, geomId = h.geomId & 0x00FFFFFFu;
    if (h.primId == 0xFFFFFFFFu) {
      memcpy(color, background, sizeof(color));
    } else if (type != LRT_TYPE_SDF_SBS_COL && type != LRT_TYPE_GRAPHICS_PRIM) {
      const uint32_t matId = mat_ids[mat_offsets[2 * geomId] + h.primId % mat_offsets[2 * geomId + 1]];
      const lrt_material* m = &materials[matId];
      if (m->type == LRT_MATERIAL_COLORED) {
        memcpy(color, m->base_color, sizeof(color));
      } else {
        color[0] = color[1] = color[2] = 0.0f;
        color[3] = 1.0f;
      }
    }
    /* rayPos = to_float3(rayPosAndNear) + to_float3(rayDirAndFar) * hit->t */
    pn[0] = pn[0] + r[4] * h.t;
    pn[1] = pn[1] + r[5] * h.t;
    pn[2] = pn[2] + r[6] * h.t;
  } while (alpha > 0.01f);
  *out = h;
  *out_tc = tc;
  *out_alpha = alpha;
  return capped;
}

/* kernel1D_FillGbufferWithTransparency (MultiRenderer.cpp:204-221): anyhit
 * per eye ray; returns how many rays reached the layer bound. */
uint64_t lrto_fill_gbuffer_transparency(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays,
                                        uint64_t n, const lrt_material* materials, const uint32_t* mat_ids,
                                        const uint32_t* mat_offsets, const float background[4], uint32_t max_layers,
                                        float* transparency, lrt_hit* hits, int threads)
{
  uint64_t capped = 0;
  (void)threads;
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 256) reduction(+ : capped)
#endif
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t cnt[LRT_COUNTER_COUNT];
    ctx_t c = {arrays, preset, cnt, 0, NULL, 0};
    f3 tc;
    float alpha;
    capped += (uint64_t)anyhit(&c, rays + 8 * i, materials, mat_ids, mat_offsets, background, max_layers, &hits[i],
                               &tc, &alpha);
    transparency[4 * i + 0] = tc.x;
    transparency[4 * i + 1] = tc.y;
    transparency[4 * i + 2] = tc.z;
    transparency[4 * i + 3] = alpha;
  }
  return capped;
}

/* MultiRenderer::Render (MultiRenderer.cpp:14-70) for one pass of
 * `samples` samples: sample s traces sample_rays[s] (n row-major eye rays
 * through initEyeRay's point s of each pixel) — through anyhit when
 * `transparency` (DIFFUSE / LAMBERT / PHONG with a transparent material),
 * blending as ResolveTransparency (MultiRenderer_resolve.cpp:573-577) — and
 * resolves with resolve_rays (sample 0's, as ResolveCommon does); the
 * colours are summed, divided by the sample count and tonemapped. */
void lrto_render_rgba8_ex(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* sample_rays,
                          uint32_t samples, const float* resolve_rays, uint64_t n, const lrt_light* lights,
                          uint32_t light_count, const float background[4], const lrt_material* materials,
                          const uint32_t* mat_ids, const uint32_t* mat_offsets, int transparency, uint32_t max_layers,
                          uint32_t* image, int threads)
{
  const uint32_t mode = preset->render_mode;
  (void)threads;
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 256)
#endif
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint64_t cnt[LRT_COUNTER_COUNT];
    float acc[4] = {0, 0, 0, 0};
    for (uint32_t smp = 0; smp < samples; smp++) {
      ctx_t c = {arrays, preset, cnt, 0, NULL, 0};
      const float* r = sample_rays + 8 * ((uint64_t)smp * n + (uint64_t)i);
      lrt_hit h;
      f3 tc = mk3(0, 0, 0);
      float alpha = 1.0f, col[4];
      if (transparency)
        anyhit(&c, r, materials, mat_ids, mat_offsets, background, max_layers, &h, &tc, &alpha);
      else
        h = nearest_hit(&c, r, r + 4);
      resolve_colour(arrays, &c, mode, h, resolve_rays + 8 * i, lights, light_count, background, materials, mat_ids,
                     mat_offsets, col);
      if (transparency) {
        col[0] = tc.x + alpha * col[0];
        col[1] = tc.y + alpha * col[1];
        col[2] = tc.z + alpha * col[2];
      }
      for (int k = 0; k < 4; k++) acc[k] = smp == 0 ? col[k] : acc[k] + col[k];
    }
    const float ns = (float)samples;
    image[i] = tonemap_rgba8(acc[0] / ns, acc[1] / ns, acc[2] / ns, acc[3] / ns);
  }
}

/* MultiRenderer::Render for OUTLINE_BORDER (MultiRenderer.cpp:55-58) over a
 * width x height image: per sample the G-buffer of that sample's rays
 * (kernel1D_FillGbuffer) and ResolveOutline (MultiRenderer_resolve.cpp:
 * 1073-1128) per pixel: the background for a miss, else white Lambert of the
 * hit shaded with the sample-0 ray, replaced by (0.2, 0.2, 0.2, 1) when the t
 * of one of the four neighbours (the pixel itself at the image's edges)
 * differs from the pixel's by more than 10 t / width; the colours are summed
 * over the samples, divided by their count and tonemapped. */
void lrto_render_outline_border(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* sample_rays,
                                uint32_t samples, const float* resolve_rays, uint32_t width, uint32_t height,
                                const lrt_light* lights, uint32_t light_count, const float background[4],
                                uint32_t* image, int threads)
{
  const uint64_t n = (uint64_t)width * height;
  lrt_hit* g = (lrt_hit*)malloc((n ? n : 1) * sizeof(lrt_hit));
  float* col = (float*)malloc((n ? n : 1) * 4 * sizeof(float));
  float* acc = (float*)calloc((n ? n : 1) * 4, sizeof(float));
  (void)threads;
  for (uint32_t smp = 0; smp < samples; smp++) {
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads > 0 ? threads : 1) schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; i++) {
      uint64_t cnt[LRT_COUNTER_COUNT];
      ctx_t c = {arrays, preset, cnt, 0, NULL, 0};
      const float* r = sample_rays + 8 * ((uint64_t)smp * n + (uint64_t)i);
      g[i] = nearest_hit(&c, r, r + 4);
      /* the Lambert colour of ResolveOutline is OUTLINE_PRIM's; resolved with
         the trace's context (a triangle's normal needs its record) */
      resolve_colour(arrays, &c, 13u, g[i], resolve_rays + 8 * i, lights, light_count, background, NULL, NULL, NULL,
                     col + 4 * i);
    }
    for (uint64_t i = 0; i < n; i++) {
      float c4[4];
      memcpy(c4, col + 4 * i, sizeof(c4));
      if (g[i].primId != 0xFFFFFFFFu) {
        const uint32_t x = (uint32_t)(i % width), y = (uint32_t)(i / width);
        const float t = g[i].t;
        const float tol = 10.0f * t / (float)width;
        const float tl = g[x == 0 ? i : i - 1].t, tu = g[y == 0 ? i : i - width].t;
        const float tr = g[x == width - 1 ? i : i + 1].t, td = g[y == height - 1 ? i : i + width].t;
        if (fabsf(tl - t) > tol || fabsf(tu - t) > tol || fabsf(tr - t) > tol || fabsf(td - t) > tol) {
          c4[0] = 0.2f;
          c4[1] = 0.2f;
          c4[2] = 0.2f;
          c4[3] = 1.0f;
        }
      }
      for (int k = 0; k < 4; k++) acc[4 * i + k] = smp == 0 ? c4[k] : acc[4 * i + k] + c4[k];
    }
  }
  const float ns = (float)samples;
  for (uint64_t i = 0; i < n; i++)
    image[i] = tonemap_rgba8(acc[4 * i] / ns, acc[4 * i + 1] / ns, acc[4 * i + 2] / ns, acc[4 * i + 3] / ns);
  free(g);
  free(col);
  free(acc);
}

void lrto_render_rgba8_modes(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays, uint64_t n,
                             const lrt_light* lights, uint32_t light_count, const float background[4],
                             const lrt_material* materials, const uint32_t* mat_ids, const uint32_t* mat_offsets,
                             uint32_t* image, int threads)
{
  lrto_render_rgba8_ex(arrays, preset, rays, 1, rays, n, lights, light_count, background, materials, mat_ids,
                       mat_offsets, 0, 256, image, threads);
}

/* rays: the eye rays of the image in row-major pixel order (initEyeRay). */
void lrto_render_rgba8(const lrt_scene_arrays* arrays, const lrt_preset* preset, const float* rays, uint64_t n,
                       const lrt_light* lights, uint32_t light_count, const float background[4], uint32_t* image,
                       int threads)
{
  lrto_render_rgba8_ex(arrays, preset, rays, 1, rays, n, lights, light_count, background, NULL, NULL, NULL, 0, 256,
                       image, threads);
}

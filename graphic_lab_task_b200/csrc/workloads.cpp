// workloads.cpp — seeded synthetic geometry for the benchmark workloads
// (declared in include/lrt_workloads.h).  Host code; no CUDA.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/lrt_workloads.h"

namespace {

// splitmix64: one 64-bit state, good enough to seed synthetic scenes.
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed ^ 0x9E3779B97F4A7C15ull) {}
  uint64_t next()
  {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
};

uint64_t hash4(int64_t x, int64_t y, int64_t z, uint64_t seed)
{
  uint64_t h = seed * 0x9E3779B97F4A7C15ull;
  h ^= uint64_t(x) * 0xC2B2AE3D27D4EB4Full;
  h = (h ^ (h >> 31)) * 0xBF58476D1CE4E5B9ull;
  h ^= uint64_t(y) * 0x165667B19E3779F9ull;
  h = (h ^ (h >> 29)) * 0x94D049BB133111EBull;
  h ^= uint64_t(z) * 0x27D4EB2F165667C5ull;
  h = (h ^ (h >> 32)) * 0xBF58476D1CE4E5B9ull;
  return h ^ (h >> 29);
}

// 3D value noise in [-1,1]: random lattice values blended with smoothstep weights.
double value_noise(double x, double y, double z, uint64_t seed)
{
  const double fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
  const int64_t ix = int64_t(fx), iy = int64_t(fy), iz = int64_t(fz);
  auto sm = [](double t) { return t * t * (3.0 - 2.0 * t); };
  const double u = sm(x - fx), v = sm(y - fy), w = sm(z - fz);
  double acc = 0.0;
  for (int c = 0; c < 8; c++) {
    const int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
    const double r = double(hash4(ix + dx, iy + dy, iz + dz, seed) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    acc += (dx ? u : 1 - u) * (dy ? v : 1 - v) * (dz ? w : 1 - w) * r;
  }
  return acc;
}

struct Sphere {
  double x, y, z, r;
};

std::vector<Sphere> load_spheres(const float* s, uint32_t n)
{
  std::vector<Sphere> v(n);
  for (uint32_t i = 0; i < n; i++) v[i] = {s[4 * i], s[4 * i + 1], s[4 * i + 2], s[4 * i + 3]};
  return v;
}

double sdf(const std::vector<Sphere>& sp, const uint32_t* ids, size_t nid, double x, double y, double z,
           uint32_t* arg = nullptr)
{
  double best = 1e30;
  uint32_t bi = 0;
  for (size_t k = 0; k < nid; k++) {
    const Sphere& s = sp[ids ? ids[k] : k];
    const double dx = x - s.x, dy = y - s.y, dz = z - s.z;
    const double d = std::sqrt(dx * dx + dy * dy + dz * dz) - s.r;
    if (d < best) { best = d; bi = ids ? ids[k] : uint32_t(k); }
  }
  if (arg) *arg = bi;
  return best;
}

// Spheres that can be the minimum anywhere inside box [lo,hi]: a sphere whose
// lower bound exceeds the smallest upper bound never wins.
void cull(const std::vector<Sphere>& sp, const double lo[3], const double hi[3], std::vector<uint32_t>& out)
{
  out.clear();
  const size_t n = sp.size();
  std::vector<double> lower(n);
  double bestUpper = 1e30;
  for (size_t i = 0; i < n; i++) {
    const Sphere& s = sp[i];
    const double c[3] = {s.x, s.y, s.z};
    double dn = 0, df = 0;
    for (int k = 0; k < 3; k++) {
      const double e = std::max({lo[k] - c[k], 0.0, c[k] - hi[k]});
      dn += e * e;
      const double f = std::max(std::fabs(c[k] - lo[k]), std::fabs(c[k] - hi[k]));
      df += f * f;
    }
    lower[i] = std::sqrt(dn) - s.r;
    bestUpper = std::min(bestUpper, std::sqrt(df) - s.r);
  }
  for (size_t i = 0; i < n; i++)
    if (lower[i] <= bestUpper + 1e-12) out.push_back(uint32_t(i));
}

uint64_t morton3(uint32_t x, uint32_t y, uint32_t z)
{
  auto spread = [](uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
  };
  return (spread(x) << 2) | (spread(y) << 1) | spread(z);
}

} // namespace

extern "C" {

lrt_status lrt_wl_noisy_sphere(uint32_t segments, float radius, float amplitude, uint64_t seed, float* verts,
                               uint32_t* tris, uint64_t* nverts, uint64_t* ntris)
{
  if (segments < 3 || !nverts || !ntris) return LRT_ERR_INVALID_ARGUMENT;
  const uint32_t rings = segments, slices = segments;
  const uint64_t nv = 2 + uint64_t(rings - 1) * slices;
  const uint64_t nt = 2ull * slices * (rings - 1);
  *nverts = nv;
  *ntris = nt;
  if (!verts || !tris) return LRT_OK;
  const double pi = 3.14159265358979323846;
  auto put = [&](uint64_t i, double nx, double ny, double nz) {
    const double disp = amplitude * value_noise(4.0 * nx + 11.0, 4.0 * ny + 17.0, 4.0 * nz + 23.0, seed);
    const double r = radius + disp;
    verts[3 * i + 0] = float(r * nx);
    verts[3 * i + 1] = float(r * ny);
    verts[3 * i + 2] = float(r * nz);
  };
  put(0, 0, 1, 0);
  for (uint32_t i = 1; i < rings; i++) {
    const double th = pi * i / rings;
    for (uint32_t j = 0; j < slices; j++) {
      const double ph = 2 * pi * j / slices;
      put(1 + uint64_t(i - 1) * slices + j, std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph));
    }
  }
  put(nv - 1, 0, -1, 0);
  uint64_t t = 0;
  auto tri = [&](uint64_t a, uint64_t b, uint64_t c) {
    tris[3 * t + 0] = uint32_t(a);
    tris[3 * t + 1] = uint32_t(b);
    tris[3 * t + 2] = uint32_t(c);
    t++;
  };
  for (uint32_t j = 0; j < slices; j++) tri(0, 1 + (j + 1) % slices, 1 + j);
  for (uint32_t i = 1; i + 1 < rings; i++) {
    const uint64_t r0 = 1 + uint64_t(i - 1) * slices, r1 = r0 + slices;
    for (uint32_t j = 0; j < slices; j++) {
      const uint64_t j1 = (j + 1) % slices;
      tri(r0 + j, r0 + j1, r1 + j);
      tri(r0 + j1, r1 + j1, r1 + j);
    }
  }
  const uint64_t last = 1 + uint64_t(rings - 2) * slices;
  for (uint32_t j = 0; j < slices; j++) tri(nv - 1, last + j, last + (j + 1) % slices);
  return t == nt ? LRT_OK : LRT_ERR_INVALID_ARGUMENT;
}

lrt_status lrt_wl_spheres(uint32_t n, float c, float rmin, float rmax, uint64_t seed, float* out)
{
  if (!out) return LRT_ERR_INVALID_ARGUMENT;
  Rng rng(seed);
  for (uint32_t i = 0; i < n; i++) {
    out[4 * i + 0] = float(rng.uniform(-c, c));
    out[4 * i + 1] = float(rng.uniform(-c, c));
    out[4 * i + 2] = float(rng.uniform(-c, c));
    out[4 * i + 3] = float(rng.uniform(rmin, rmax));
  }
  return LRT_OK;
}

double lrt_wl_sphere_sdf(const float* s, uint32_t n, double x, double y, double z)
{
  return sdf(load_spheres(s, n), nullptr, n, x, y, z);
}

lrt_status lrt_wl_sbs_from_spheres(const float* s4, uint32_t n, uint32_t grid_res, uint32_t bs, uint32_t pad,
                                   lrt_sdf_sbs_header* header, lrt_sdf_sbs_node* nodes, uint32_t* values,
                                   float* values_f, uint64_t* node_count, uint64_t* values_count,
                                   uint64_t* values_f_count)
{
  if (!s4 || n == 0 || bs == 0 || grid_res % bs != 0 || !node_count || !values_count || !values_f_count)
    return LRT_ERR_INVALID_ARGUMENT;
  const uint32_t G = grid_res / bs;
  if (G > 0xFFFF) return LRT_ERR_INVALID_ARGUMENT;
  const auto sp = load_spheres(s4, n);
  const double vox = 2.0 / grid_res;
  const double diag = std::sqrt(3.0) * bs * vox;
  const uint32_t v = bs + 2 * pad + 1;
  const uint64_t v3 = uint64_t(v) * v * v;

  // bricks in Morton order so that neighbouring bricks sit close in memory
  std::vector<uint64_t> order(uint64_t(G) * G * G);
  for (uint32_t x = 0; x < G; x++)
    for (uint32_t y = 0; y < G; y++)
      for (uint32_t z = 0; z < G; z++) order[(uint64_t(x) * G + y) * G + z] = (morton3(x, y, z) << 24) | 0;
  std::vector<uint8_t> keep(order.size());
#pragma omp parallel
  {
    std::vector<uint32_t> ids;
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < int64_t(order.size()); i++) {
      const uint32_t x = uint32_t(i / (uint64_t(G) * G)), y = uint32_t((i / G) % G), z = uint32_t(i % G);
      const double lo[3] = {-1 + vox * x * bs, -1 + vox * y * bs, -1 + vox * z * bs};
      const double hi[3] = {lo[0] + vox * bs, lo[1] + vox * bs, lo[2] + vox * bs};
      cull(sp, lo, hi, ids);
      bool k = false;
      for (int c = 0; c < 8 && !k; c++) {
        const double d = sdf(sp, ids.data(), ids.size(), (c & 4) ? hi[0] : lo[0], (c & 2) ? hi[1] : lo[1],
                             (c & 1) ? hi[2] : lo[2]);
        k = std::fabs(d) < diag;
      }
      keep[i] = k;
    }
  }
  std::vector<std::pair<uint64_t, uint32_t>> kept; // (morton, linear)
  for (uint64_t i = 0; i < order.size(); i++)
    if (keep[i]) {
      const uint32_t x = uint32_t(i / (uint64_t(G) * G)), y = uint32_t((i / G) % G), z = uint32_t(i % G);
      kept.push_back({morton3(x, y, z), uint32_t(i)});
    }
  std::sort(kept.begin(), kept.end());
  const uint64_t nb = kept.size();
  *node_count = nb;
  *values_count = nb * (v3 + 8);
  *values_f_count = 3ull * n + nb * v3;
  if (!header || !nodes || !values || !values_f) return LRT_OK;

  header->brick_size = bs;
  header->brick_pad = pad;
  header->bytes_per_value = 4;
  header->aux_data = LRT_SBS_LAYOUT_ID32F_IRGB32F;
  Rng crng(0xC0105ull);
  for (uint32_t i = 0; i < n; i++)
    for (int k = 0; k < 3; k++) values_f[3 * i + k] = float(0.2 + 0.8 * crng.uniform());

#pragma omp parallel
  {
    std::vector<uint32_t> ids;
#pragma omp for schedule(dynamic, 16)
    for (int64_t k = 0; k < int64_t(nb); k++) {
      const uint32_t i = kept[k].second;
      const uint32_t x = uint32_t(i / (uint64_t(G) * G)), y = uint32_t((i / G) % G), z = uint32_t(i % G);
      lrt_sdf_sbs_node& nd = nodes[k];
      nd.pos_xy = (x << 16) | y;
      nd.pos_z_lod_size = (z << 16) | G;
      nd.data_offset = uint32_t(uint64_t(k) * (v3 + 8));
      nd._pad = 0;
      const double org[3] = {-1 + vox * (double(x) * bs - pad), -1 + vox * (double(y) * bs - pad),
                             -1 + vox * (double(z) * bs - pad)};
      const double lo[3] = {org[0], org[1], org[2]};
      const double hi[3] = {org[0] + vox * (v - 1), org[1] + vox * (v - 1), org[2] + vox * (v - 1)};
      cull(sp, lo, hi, ids);
      uint32_t* vals = values + uint64_t(k) * (v3 + 8);
      float* vf = values_f + 3ull * n + uint64_t(k) * v3;
      const uint32_t fbase = uint32_t(3ull * n + uint64_t(k) * v3);
      for (uint32_t a = 0; a < v; a++)
        for (uint32_t b = 0; b < v; b++)
          for (uint32_t c = 0; c < v; c++) {
            const uint32_t vid = (a * v + b) * v + c;
            vf[vid] = float(sdf(sp, ids.data(), ids.size(), org[0] + vox * a, org[1] + vox * b, org[2] + vox * c));
            vals[vid] = fbase + vid;
          }
      for (int c = 0; c < 8; c++) {
        uint32_t arg = 0;
        const double px = -1 + vox * (double(x) * bs + ((c & 4) ? bs : 0));
        const double py = -1 + vox * (double(y) * bs + ((c & 2) ? bs : 0));
        const double pz = -1 + vox * (double(z) * bs + ((c & 1) ? bs : 0));
        sdf(sp, nullptr, sp.size(), px, py, pz, &arg);
        vals[v3 + c] = 3 * arg;
      }
    }
  }
  return LRT_OK;
}

lrt_status lrt_wl_frame_octree_from_spheres(const float* s4, uint32_t n, uint32_t max_depth,
                                            lrt_sdf_frame_octree_node* out, uint64_t* node_count)
{
  if (!s4 || !node_count || max_depth > 16) return LRT_ERR_INVALID_ARGUMENT;
  const auto sp = load_spheres(s4, n);
  struct Cell {
    uint32_t px, py, pz, level;
  };
  std::vector<Cell> cells;
  std::vector<lrt_sdf_frame_octree_node> nodes;
  cells.push_back({0, 0, 0, 0});
  nodes.push_back(lrt_sdf_frame_octree_node{});
  std::vector<uint32_t> ids;
  for (size_t i = 0; i < cells.size(); i++) {
    const Cell c = cells[i];
    const double d = 1.0 / double(1u << c.level); // fraction of the unit cube
    const double lo[3] = {2 * d * c.px - 1, 2 * d * c.py - 1, 2 * d * c.pz - 1};
    const double hi[3] = {lo[0] + 2 * d, lo[1] + 2 * d, lo[2] + 2 * d};
    cull(sp, lo, hi, ids);
    for (int k = 0; k < 8; k++)
      nodes[i].values[k] = float(sdf(sp, ids.data(), ids.size(), (k & 4) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1],
                                     (k & 1) ? hi[2] : lo[2]));
    nodes[i].offset = 0;
    const double centre = sdf(sp, ids.data(), ids.size(), lo[0] + d, lo[1] + d, lo[2] + d);
    if (c.level < max_depth && std::fabs(centre) < std::sqrt(3.0) * d) {
      nodes[i].offset = uint32_t(nodes.size());
      for (int k = 0; k < 8; k++) {
        cells.push_back({2 * c.px + ((k & 4) >> 2), 2 * c.py + ((k & 2) >> 1), 2 * c.pz + (k & 1), c.level + 1});
        nodes.push_back(lrt_sdf_frame_octree_node{});
      }
    }
  }
  *node_count = nodes.size();
  if (out) std::memcpy(out, nodes.data(), nodes.size() * sizeof(nodes[0]));
  return LRT_OK;
}

lrt_status lrt_wl_svs_from_spheres(const float* s4, uint32_t n, uint32_t lod, lrt_sdf_svs_node* out,
                                   uint64_t* node_count)
{
  if (!s4 || !node_count || lod > 15) return LRT_ERR_INVALID_ARGUMENT;
  const auto sp = load_spheres(s4, n);
  const uint32_t N = 1u << lod;
  const double dmax = 2 * 1.73205081 / N;
  std::vector<lrt_sdf_svs_node> nodes;
  std::vector<uint32_t> ids;
  struct Cell {
    uint32_t px, py, pz, level;
  };
  std::vector<Cell> stack{{0, 0, 0, 0}};
  while (!stack.empty()) {
    const Cell c = stack.back();
    stack.pop_back();
    const double d = 1.0 / double(1u << c.level);
    const double lo[3] = {2 * d * c.px - 1, 2 * d * c.py - 1, 2 * d * c.pz - 1};
    const double hi[3] = {lo[0] + 2 * d, lo[1] + 2 * d, lo[2] + 2 * d};
    cull(sp, lo, hi, ids);
    const double centre = sdf(sp, ids.data(), ids.size(), lo[0] + d, lo[1] + d, lo[2] + d);
    if (std::fabs(centre) >= std::sqrt(3.0) * d) continue;
    if (c.level < lod) {
      for (int k = 7; k >= 0; k--)
        stack.push_back({2 * c.px + ((k & 4) >> 2), 2 * c.py + ((k & 2) >> 1), 2 * c.pz + (k & 1), c.level + 1});
      continue;
    }
    bool less = false, more = false;
    uint32_t q[8];
    for (int k = 0; k < 8; k++) {
      const double v = sdf(sp, ids.data(), ids.size(), (k & 4) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1],
                           (k & 1) ? hi[2] : lo[2]);
      if (v <= 0) less = true; else more = true;
      const double qq = std::round((v + dmax) / (2 * dmax) * 255.0);
      q[k] = uint32_t(std::min(255.0, std::max(0.0, qq)));
    }
    if (!(less && more)) continue;
    lrt_sdf_svs_node nd;
    nd.pos_xy = (c.px << 16) | c.py;
    nd.pos_z_lod_size = (c.pz << 16) | N;
    nd.values[0] = q[0] | (q[1] << 8) | (q[2] << 16) | (q[3] << 24);
    nd.values[1] = q[4] | (q[5] << 8) | (q[6] << 16) | (q[7] << 24);
    nodes.push_back(nd);
  }
  *node_count = nodes.size();
  if (out) std::memcpy(out, nodes.data(), nodes.size() * sizeof(nodes[0]));
  return LRT_OK;
}

} // extern "C"

// layout.cpp — builds the derived device layouts of device_layout.h on the
// host (compiled with -ffp-contract=off so every float is computed exactly
// as the reference computes it on the fly).
#include <algorithm>
#include <cstring>

#include "layout.h"

namespace lrt {

void build_geoms(const HostArrays& h, std::vector<DevGeom>& out)
{
  out.resize(h.geomData.size());
  for (size_t g = 0; g < h.geomData.size(); g++) {
    const lrt_geom_data& gd = h.geomData[g];
    DevGeom d;
    std::memset(&d, 0, sizeof(d));
    d.tag = h.geomTags[g];
    d.type = gd.type;
    d.bvhOffset = gd.bvhOffset;
    d.aabbBase = h.startEnd[2 * g];
    if (d.tag == LRT_TAG_TRIANGLE) {
      d.triBase = gd.offset[0] / 3;
    } else {
      d.sdfId = gd.offset[0];
      if (d.tag == LRT_TAG_SDF_BRICK) d.sdfRoot = h.sdfSBSRoots[d.sdfId];
      else if (gd.type == LRT_TYPE_SDF_FRAME_OCTREE) d.sdfRoot = h.sdfFrameOctreeRoots[d.sdfId];
      else if (gd.type == LRT_TYPE_SDF_SVS) d.sdfRoot = h.sdfSVSRoots[d.sdfId];
    }
    out[g] = d;
  }
}

// {A, B-A, C-A} per reordered triangle slot; IntersectAllTrianglesInLeaf
// computes exactly these differences (BVH2Common.cpp:1585-1589).
void build_tri_soup(const HostArrays& h, std::vector<float>& soup)
{
  const size_t nslots = h.indices.size() / 3;
  soup.assign(nslots * 12, 0.0f);
  for (size_t g = 0; g < h.geomData.size(); g++) {
    if (h.geomTags[g] != LRT_TAG_TRIANGLE) continue;
    const lrt_geom_data& gd = h.geomData[g];
    uint64_t ntri = 0;
    for (uint32_t a = h.startEnd[2 * g]; a < h.startEnd[2 * g + 1]; a++) {
      const uint32_t pk = h.primIdCount[a];
      ntri = std::max<uint64_t>(ntri, uint64_t(pk & 0x0FFFFFFFu) + ((pk & 0x70000000u) >> 28));
    }
    const uint64_t base = gd.offset[0] / 3;
    for (uint64_t t = 0; t < ntri && base + t < nslots; t++) {
      const float* P[3];
      for (int c = 0; c < 3; c++) P[c] = h.vertPos.data() + 4 * (uint64_t(gd.offset[1]) + h.indices[gd.offset[0] + 3 * t + c]);
      float* o = soup.data() + 12 * (base + t);
      for (int k = 0; k < 3; k++) {
        o[k] = P[0][k];
        o[4 + k] = P[1][k] - P[0][k];
        o[8 + k] = P[2][k] - P[0][k];
      }
    }
  }
}

// Dense (brick_size+1)^3 corner grids per SBS node; values as
// load_distance_values returns them (BVH2Common.cpp:846-882).
void build_sbs_dense(const HostArrays& h, std::vector<DevSbs>& sbs, std::vector<float>& dense)
{
  const size_t nsdf = h.sdfSBSRoots.size();
  sbs.assign(nsdf, DevSbs{});
  uint64_t total = 0;
  std::vector<uint64_t> counts(nsdf);
  for (size_t i = 0; i < nsdf; i++) {
    const uint32_t root = h.sdfSBSRoots[i];
    uint64_t next = h.sdfSBSNodes.size();
    for (size_t j = 0; j < nsdf; j++)
      if (h.sdfSBSRoots[j] > root) next = std::min<uint64_t>(next, h.sdfSBSRoots[j]);
    counts[i] = next > root ? next - root : 0;
    const lrt_sdf_sbs_header& hd = h.sdfSBSHeaders[i];
    const uint32_t V1 = hd.brick_size + 1;
    const uint32_t v = hd.brick_size + 2 * hd.brick_pad + 1;
    DevSbs& d = sbs[i];
    d.nodeCount = uint32_t(counts[i]);
    d.denseBase = total;
    d.denseStride = V1 * V1 * V1;
    d.brick_size = hd.brick_size;
    d.v3 = v * v * v;
    const uint32_t layout = hd.aux_data & LRT_SBS_LAYOUT_MASK;
    d.colorLayout = (layout == LRT_SBS_LAYOUT_ID32F_IRGB32F || layout == LRT_SBS_LAYOUT_ID32F_IRGB32F_IN) ? 1u : 0u;
    total += counts[i] * d.denseStride;
  }
  dense.assign(total, 0.0f);
  for (size_t i = 0; i < nsdf; i++) {
    const lrt_sdf_sbs_header& hd = h.sdfSBSHeaders[i];
    const DevSbs& d = sbs[i];
    const uint32_t bs = hd.brick_size, pad = hd.brick_pad, V1 = bs + 1;
    const uint32_t v = bs + 2 * pad + 1;
    const bool indexed = d.colorLayout != 0;
    const uint32_t vals_per_int = indexed ? 1 : 4 / hd.bytes_per_value;
    const uint32_t bits = indexed ? 32 : 8 * hd.bytes_per_value;
    const uint32_t max_val = (!indexed && hd.bytes_per_value != 4) ? ((1u << bits) - 1) : 0xFFFFFFFFu;
    const uint32_t root = h.sdfSBSRoots[i];
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < int64_t(counts[i]); k++) {
      const lrt_sdf_sbs_node& nd = h.sdfSBSNodes[root + k];
      const uint32_t off = nd.data_offset;
      float* o = dense.data() + d.denseBase + uint64_t(k) * d.denseStride;
      const float sz = float(nd.pos_z_lod_size & 0x0000FFFF);
      const float sz_inv = 2.0f / sz;
      const float d_max = 1.73205081f * sz_inv;
      const float mult = 2 * d_max / max_val;
      for (uint32_t x = 0; x < V1; x++)
        for (uint32_t y = 0; y < V1; y++)
          for (uint32_t z = 0; z < V1; z++) {
            const uint32_t vId = (x + pad) * v * v + (y + pad) * v + (z + pad);
            float val;
            if (indexed) {
              val = h.sdfSBSDataF[h.sdfSBSData[off + vId]];
            } else {
              const uint32_t word = h.sdfSBSData[off + vId / vals_per_int];
              const uint32_t sh = bits * (vId % vals_per_int);
              const uint32_t field = (sh >= 32 ? 0u : (word >> sh)) & max_val;
              val = -d_max + mult * field;
            }
            o[(x * V1 + y) * V1 + z] = val;
          }
    }
  }
}

} // namespace lrt

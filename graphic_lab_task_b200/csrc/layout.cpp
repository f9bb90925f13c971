// layout.cpp — builds the derived device layouts of device_layout.h on the
// host (compiled with -ffp-contract=off so every float is computed exactly
// as the reference computes it on the fly).
#include <algorithm>
#include <cstring>
#include <functional>
#include <limits>

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

// Surface-voxel masks of every brick from its dense corner grid (see
// device_layout.h): vmin is reduced exactly as load_distance_values does
// (BVH2Common.cpp:861-866), so the bit equals the reference's `vmin <= 0`.
void build_sbs_masks(const HostArrays& h, std::vector<DevSbs>& sbs, const std::vector<float>& dense,
                     std::vector<uint32_t>& mask)
{
  uint64_t total = 0;
  for (size_t i = 0; i < sbs.size(); i++) {
    const uint32_t bs = sbs[i].brick_size;
    sbs[i].maskStride = 1 + (bs * bs * bs + 31) / 32;
    sbs[i].maskBase = total;
    total += uint64_t(sbs[i].nodeCount) * sbs[i].maskStride;
  }
  mask.assign(total, 0u);
  for (size_t i = 0; i < sbs.size(); i++) {
    const DevSbs& d = sbs[i];
    const uint32_t bs = d.brick_size, V1 = bs + 1;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < int64_t(d.nodeCount); k++) {
      const float* g = dense.data() + d.denseBase + uint64_t(k) * d.denseStride;
      uint32_t* m = mask.data() + d.maskBase + uint64_t(k) * d.maskStride;
      for (uint32_t x = 0; x < bs; x++)
        for (uint32_t y = 0; y < bs; y++)
          for (uint32_t z = 0; z < bs; z++) {
            float vmin = 1e6f;
            for (int c = 0; c < 8; c++) {
              const float v = g[((x + ((c & 4) >> 2)) * V1 + (y + ((c & 2) >> 1))) * V1 + (z + (c & 1))];
              vmin = (v < vmin) ? v : vmin;
            }
            if (vmin <= 0.0f) {
              const uint32_t vid = (x * bs + y) * bs + z;
              m[1 + vid / 32] |= 1u << (vid % 32);
              m[0] = 1;
            }
          }
    }
  }
  (void)h;
}

// Device copy of the BLAS node pairs in which every child subtree of an SBS
// BLAS that holds no brick able to start a sphere trace gets a NaN box.  A
// NaN box fails the child test of BVH2TraverseF32 (tmin <= tmax is false) for
// every ray, so such a subtree is never entered.  This cannot change a
// result: the pruned leaves never touch the hit, and the depth-first
// near-first order of the remaining leaves is unchanged — at a node whose
// other child is pruned the reference would visit that child (before or
// after) without effect.  Returns the number of pruned children.
uint64_t prune_sbs_pairs(const HostArrays& h, const std::vector<DevGeom>& geoms, const std::vector<DevSbs>& sbs,
                         const std::vector<uint32_t>& mask, std::vector<lrt_bvh_node_pair>& pairs)
{
  pairs = h.allNodePairs;
  const float qnan = std::numeric_limits<float>::quiet_NaN();
  uint64_t pruned = 0;
  for (size_t g = 0; g < geoms.size(); g++) {
    if (geoms[g].tag != LRT_TAG_SDF_BRICK) continue;
    const DevSbs& sb = sbs[geoms[g].sdfId];
    const uint32_t base = geoms[g].bvhOffset, a0 = geoms[g].aabbBase;
    // returns true if the subtree under `lo` (a child word) can produce a hit
    std::function<bool(uint32_t)> live = [&](uint32_t lo) -> bool {
      if (lo & kLeafBit) {
        if (lo == kLeafNormal) return false;
        const uint32_t primId = h.primIdCount[a0 + (lo & kStartMask)] & kStartMask;
        if (primId >= sb.nodeCount) return false;
        return mask[sb.maskBase + uint64_t(primId) * sb.maskStride] != 0;
      }
      lrt_bvh_node_pair& p = pairs[base + lo];
      const bool l = live(p.left.leftOffset), r = live(p.right.leftOffset);
      for (int j = 0; j < 2; j++) {
        lrt_bvh_node& n = j ? p.right : p.left;
        if (!(j ? r : l)) {
          for (int k = 0; k < 3; k++) n.boxMin[k] = n.boxMax[k] = qnan;
          pruned++;
        }
      }
      return l || r;
    };
    live(0); // the root pair
  }
  return pruned;
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
    d.pad = hd.brick_pad;
    d.vsize = v;
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

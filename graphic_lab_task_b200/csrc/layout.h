// layout.h — host builders of the derived device layouts (layout.cpp).
#pragma once
#include <vector>

#include "device_layout.h"
#include "scene.h"

namespace lrt {

void build_geoms(const HostArrays& h, std::vector<DevGeom>& out);
void build_tri_soup(const HostArrays& h, std::vector<float>& soup);
void build_sbs_dense(const HostArrays& h, std::vector<DevSbs>& sbs, std::vector<float>& dense);
void build_sbs_masks(const HostArrays& h, std::vector<DevSbs>& sbs, const std::vector<float>& dense,
                     std::vector<uint32_t>& mask);
uint64_t prune_sbs_pairs(const HostArrays& h, const std::vector<DevGeom>& geoms, const std::vector<DevSbs>& sbs,
                         const std::vector<uint32_t>& mask, std::vector<lrt_bvh_node_pair>& pairs);

} // namespace lrt

// layout.h — host builders of the derived device layouts (layout.cpp).
#pragma once
#include <vector>

#include "device_layout.h"
#include "scene.h"

namespace lrt {

void build_geoms(const HostArrays& h, std::vector<DevGeom>& out);
void build_tri_soup(const HostArrays& h, std::vector<float>& soup);
void build_sbs_dense(const HostArrays& h, std::vector<DevSbs>& sbs, std::vector<float>& dense);

} // namespace lrt

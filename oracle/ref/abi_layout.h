// abi_layout.h — the C-ABI's POD structs (include/lrt_b200.h) against the
// reference's own definitions, field by field: same size and the same offset
// for every field, so that the reference's arrays can be handed to the
// library by pointer and its preset copied byte for byte.
//
// TEST INFRASTRUCTURE ONLY: included by the checker (ref_harness.cpp) and by
// the compiled drop-in subclass (bvhrt_b200.cpp), both built against the
// reference's headers.
#pragma once
#include <cstddef>

#include "MultiRenderer/BVH2Common.h"
#include "core/IRenderer.h"

#include "../../include/lrt_b200.h"

#define LRT_SAME_FIELD(R, O, rf, of) \
  static_assert(offsetof(R, rf) == offsetof(O, of), #R "::" #rf " at the offset of " #O "::" #of)
#define LRT_SAME_SIZE(R, O) static_assert(sizeof(R) == sizeof(O), "sizeof(" #R ") == sizeof(" #O ")")

// CRT_Hit, CrossRT/CrossRT.h:26-33
LRT_SAME_SIZE(CRT_Hit, lrt_hit);
LRT_SAME_FIELD(CRT_Hit, lrt_hit, t, t);
LRT_SAME_FIELD(CRT_Hit, lrt_hit, primId, primId);
LRT_SAME_FIELD(CRT_Hit, lrt_hit, instId, instId);
LRT_SAME_FIELD(CRT_Hit, lrt_hit, geomId, geomId);
LRT_SAME_FIELD(CRT_Hit, lrt_hit, coords, coords);

// BVHNode / BVHNodePair, utils/raytracing/cbvh.h:21-33
LRT_SAME_SIZE(BVHNode, lrt_bvh_node);
LRT_SAME_FIELD(BVHNode, lrt_bvh_node, boxMin, boxMin);
LRT_SAME_FIELD(BVHNode, lrt_bvh_node, leftOffset, leftOffset);
LRT_SAME_FIELD(BVHNode, lrt_bvh_node, boxMax, boxMax);
LRT_SAME_FIELD(BVHNode, lrt_bvh_node, escapeIndex, escapeIndex);
LRT_SAME_SIZE(BVHNodePair, lrt_bvh_node_pair);
LRT_SAME_FIELD(BVHNodePair, lrt_bvh_node_pair, left, left);
LRT_SAME_FIELD(BVHNodePair, lrt_bvh_node_pair, right, right);

// GeomData / InstanceData, utils/raytracing/intersection_common.h:33-56
LRT_SAME_SIZE(GeomData, lrt_geom_data);
LRT_SAME_FIELD(GeomData, lrt_geom_data, boxMin, boxMin);
LRT_SAME_FIELD(GeomData, lrt_geom_data, boxMax, boxMax);
LRT_SAME_FIELD(GeomData, lrt_geom_data, bvhOffset, bvhOffset);
LRT_SAME_FIELD(GeomData, lrt_geom_data, type, type);
LRT_SAME_FIELD(GeomData, lrt_geom_data, offset, offset);
LRT_SAME_FIELD(GeomData, lrt_geom_data, hasChannels, hasChannels);
LRT_SAME_FIELD(GeomData, lrt_geom_data, _pad, _pad);
LRT_SAME_SIZE(InstanceData, lrt_instance_data);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, boxMin, boxMin);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, boxMax, boxMax);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, geomId, geomId);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, _pad, _pad);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, transform, transform);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, transformInv, transformInv);
LRT_SAME_FIELD(InstanceData, lrt_instance_data, transformInvTransposed, transformInvTransposed);

// SDF nodes and header, sdf/simple/sdf_simple_shared.h:23-55
LRT_SAME_SIZE(SdfFrameOctreeNode, lrt_sdf_frame_octree_node);
LRT_SAME_FIELD(SdfFrameOctreeNode, lrt_sdf_frame_octree_node, values, values);
LRT_SAME_FIELD(SdfFrameOctreeNode, lrt_sdf_frame_octree_node, offset, offset);
LRT_SAME_SIZE(SdfSVSNode, lrt_sdf_svs_node);
LRT_SAME_FIELD(SdfSVSNode, lrt_sdf_svs_node, pos_xy, pos_xy);
LRT_SAME_FIELD(SdfSVSNode, lrt_sdf_svs_node, pos_z_lod_size, pos_z_lod_size);
LRT_SAME_FIELD(SdfSVSNode, lrt_sdf_svs_node, values, values);
LRT_SAME_SIZE(SdfSBSNode, lrt_sdf_sbs_node);
LRT_SAME_FIELD(SdfSBSNode, lrt_sdf_sbs_node, pos_xy, pos_xy);
LRT_SAME_FIELD(SdfSBSNode, lrt_sdf_sbs_node, pos_z_lod_size, pos_z_lod_size);
LRT_SAME_FIELD(SdfSBSNode, lrt_sdf_sbs_node, data_offset, data_offset);
LRT_SAME_FIELD(SdfSBSNode, lrt_sdf_sbs_node, _pad, _pad);
LRT_SAME_SIZE(SdfSBSHeader, lrt_sdf_sbs_header);
LRT_SAME_FIELD(SdfSBSHeader, lrt_sdf_sbs_header, brick_size, brick_size);
LRT_SAME_FIELD(SdfSBSHeader, lrt_sdf_sbs_header, brick_pad, brick_pad);
LRT_SAME_FIELD(SdfSBSHeader, lrt_sdf_sbs_header, bytes_per_value, bytes_per_value);
LRT_SAME_FIELD(SdfSBSHeader, lrt_sdf_sbs_header, aux_data, aux_data);

// MultiRenderPreset, core/render_settings.h:116-137
LRT_SAME_SIZE(MultiRenderPreset, lrt_preset);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, render_mode, render_mode);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, sdf_node_intersect, sdf_node_intersect);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, normal_mode, normal_mode);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, ray_gen_mode, ray_gen_mode);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, interpolation_mode, interpolation_mode);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, representation_mode, representation_mode);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, spp, spp);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, fixed_lod, fixed_lod);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, level_of_detail, level_of_detail);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, compact_sdf_eps, compact_sdf_eps);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, LOD_distance, LOD_distance);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, channel_render_mode, channel_render_mode);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, channel_id, channel_id);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, component_id, component_id);
LRT_SAME_FIELD(MultiRenderPreset, lrt_preset, CTF_id, CTF_id);

// Light and MultiRendererMaterial, core/IRenderer.h:32-39, 72-78
LRT_SAME_SIZE(Light, lrt_light);
LRT_SAME_FIELD(Light, lrt_light, space, space);
LRT_SAME_FIELD(Light, lrt_light, type, type);
LRT_SAME_FIELD(Light, lrt_light, color, color);
LRT_SAME_FIELD(Light, lrt_light, _pad, _pad);
LRT_SAME_SIZE(MultiRendererMaterial, lrt_material);
LRT_SAME_FIELD(MultiRendererMaterial, lrt_material, type, type);
LRT_SAME_FIELD(MultiRendererMaterial, lrt_material, texId, texId);
LRT_SAME_FIELD(MultiRendererMaterial, lrt_material, metallic, metallic);
LRT_SAME_FIELD(MultiRendererMaterial, lrt_material, roughness, roughness);
LRT_SAME_FIELD(MultiRendererMaterial, lrt_material, base_color, base_color);

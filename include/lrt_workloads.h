/*
 * lrt_workloads.h — seeded synthetic geometry for the benchmark workloads
 * (part of liblrt_b200.so).  Not a reference interface: these generators
 * produce the inputs the reference's own builders would take
 * (a triangle soup for AddGeom_Triangles3f, SdfSBS / frame-octree / SVS
 * models for AddGeom_Sdf*), in the reference's data formats
 * (sdf/simple/sdf_simple_shared.h).
 *
 * Every generator is deterministic for a given seed.  Two-phase calls: pass
 * NULL output pointers to receive the sizes, then call again with buffers.
 */
#ifndef LRT_WORKLOADS_H
#define LRT_WORKLOADS_H

#include <stddef.h>
#include <stdint.h>

#include "lrt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* UV sphere with `segments` latitude rings and longitude slices
 * (2*segments*(segments-1) triangles), every vertex displaced along its
 * normal by amplitude * value_noise(p) (seeded 3D value noise in [-1,1]).
 * verts: nverts*3 floats, tris: ntris*3 uint32. */
lrt_status lrt_wl_noisy_sphere(uint32_t segments, float radius, float amplitude, uint64_t seed, float* verts,
                               uint32_t* tris, uint64_t* nverts, uint64_t* ntris);

/* n spheres {cx, cy, cz, r}: centres U[-c,c]^3, radii U[rmin,rmax]. */
lrt_status lrt_wl_spheres(uint32_t n, float c, float rmin, float rmax, uint64_t seed, float* out4n);

/* Signed distance of the union (min) of the spheres at one point (double). */
double lrt_wl_sphere_sdf(const float* spheres4n, uint32_t n, double x, double y, double z);

/* Sparse brick set of the sphere-union SDF sampled on a virtual
 * grid_res^3 grid over [-1,1]^3, bricks of brick_size^3 voxels with
 * brick_pad border voxels, layout SDF_SBS_NODE_LAYOUT_ID32F_IRGB32F
 * (fp32 distances through indices, 8 colour indices per brick).  A brick is
 * kept iff |d| < brick diagonal at one of its 8 corners.
 * values_f starts with a palette of 3 floats per sphere (corner colour = colour
 * of the nearest sphere), then (brick_size+2*pad+1)^3 distances per brick.
 * values per brick: v^3 indices into values_f, then 8 colour indices. */
lrt_status lrt_wl_sbs_from_spheres(const float* spheres4n, uint32_t n, uint32_t grid_res, uint32_t brick_size,
                                   uint32_t brick_pad, lrt_sdf_sbs_header* header, lrt_sdf_sbs_node* nodes,
                                   uint32_t* values, float* values_f, uint64_t* node_count, uint64_t* values_count,
                                   uint64_t* values_f_count);

/* Frame octree of the sphere-union SDF over [-1,1]^3: a node is split
 * (8 children stored consecutively) while depth < max_depth and
 * |d(centre)| < half its diagonal; values are the distances at the 8 corners. */
lrt_status lrt_wl_frame_octree_from_spheres(const float* spheres4n, uint32_t n, uint32_t max_depth,
                                            lrt_sdf_frame_octree_node* nodes, uint64_t* node_count);

/* Sparse voxel set at level `lod` (2^lod voxels per side): voxels whose
 * 8 corner distances change sign, quantised to 8 bits with
 * d_max = 2*sqrt(3)/2^lod (the dequantisation of BVH2Common.cpp:200-203). */
lrt_status lrt_wl_svs_from_spheres(const float* spheres4n, uint32_t n, uint32_t lod, lrt_sdf_svs_node* nodes,
                                   uint64_t* node_count);

#ifdef __cplusplus
}
#endif
#endif /* LRT_WORKLOADS_H */

// link_stubs.cpp — definitions that let the reference's BVHRT host code
// (MultiRenderer/BVH2Common_host.cpp) and MultiRenderer
// (MultiRenderer/MultiRenderer*.cpp) link without their scene-file I/O,
// mesh-file, compression and scene-graph libraries.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle/_ref checker build).  The ray
// query and render paths never reach any of these: they back
// AddCustomGeom_FromFile, the compressed-octree adders, LiteScene XML nodes,
// MultiRenderer::LoadScene and the data-channel (CAE) modes.  Each one aborts
// with a message if it is ever called, so a silent wrong result is
// impossible.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "LiteScene/hydraxml.h"
#include "LiteScene/scene.h"
#include "sdf/multi/sdf_multi.h"
#include "sdf/scom/scom.h"
#include "sdf/scom/similarity_compression.h"
#include "sdf/scom2/clustering/symmetric_groups.h"
#include "sdf/scom2/scom.h"
#include "sdf/simple/sdf_simple.h"
#include "utils/common/data_channel.h"
#include "utils/common/strings.h"
#include "utils/mesh/augmented_mesh.h"
#include "utils/mesh/mesh.h"
#include "utils/mesh/mesh_internal.h"

[[noreturn]] static void off_path(const char* what)
{
  std::fprintf(stderr, "liblrt_ref: %s is outside the ray-query path and is not linked\n", what);
  std::abort();
}

namespace LiteScene {
bool Geometry::load_node_base(pugi::xml_node) { off_path("Geometry::load_node_base"); }
void Geometry::save_node_base(pugi::xml_node&) const { off_path("Geometry::save_node_base"); }
bool CustomGeometry::load_node(pugi::xml_node) { off_path("CustomGeometry::load_node"); }
bool CustomGeometry::save_node(pugi::xml_node&) const { off_path("CustomGeometry::save_node"); }
bool CustomGeometry::load_data(const SceneMetadata&) { off_path("CustomGeometry::load_data"); }
bool CustomGeometry::save_data(const SceneMetadata&) { off_path("CustomGeometry::save_data"); }
std::wstring s2ws(const std::string&) { off_path("LiteScene::s2ws"); }
std::string ws2s(const std::wstring&) { off_path("LiteScene::ws2s"); }
bool MeshGeometry::load_node(pugi::xml_node) { off_path("MeshGeometry::load_node"); }
bool MeshGeometry::save_node(pugi::xml_node&) const { off_path("MeshGeometry::save_node"); }
bool MeshGeometry::load_data(const SceneMetadata&) { off_path("MeshGeometry::load_data"); }
bool MeshGeometry::save_data(const SceneMetadata&) { off_path("MeshGeometry::save_data"); }
bool HydraScene::load(const std::string&) { off_path("HydraScene::load"); }
void HydraScene::initialize_empty_scene() { off_path("HydraScene::initialize_empty_scene"); }
void HydraScene::clear() { off_path("HydraScene::clear"); }
} // namespace LiteScene

DataChannelInfo get_info(const DataChannel&) { off_path("get_info(DataChannel)"); }
std::vector<std::string> split(const std::string&, char) { off_path("split"); }

namespace cmesh4 {
void save_augmented_mesh(const AugmentedMesh&, const char*) { off_path("cmesh4::save_augmented_mesh"); }
void recalculate_vertex_normals(SimpleMesh&) { off_path("cmesh4::recalculate_vertex_normals"); }
void load_augmented_mesh(AugmentedMesh&, const char*) { off_path("cmesh4::load_augmented_mesh"); }
void fix_missing(SimpleMesh&, int) { off_path("cmesh4::fix_missing"); }
} // namespace cmesh4

void save_coctree_v3(const COctreeV3View&, const std::string&) { off_path("save_coctree_v3"); }
void load_coctree_v3(COctreeV3&, const std::string&) { off_path("load_coctree_v3"); }
void save_scom2(const SCom2Tree&, const std::string&) { off_path("save_scom2"); }
void load_scom2(SCom2Tree&, const std::string&) { off_path("load_scom2"); }
void save_sdf_DAG(const SdfDAG&, const std::string&) { off_path("save_sdf_DAG"); }
void load_sdf_DAG(SdfDAG&, const std::string&) { off_path("load_sdf_DAG"); }
void save_sdf_multi_octree(const SdfMultiOctreeView&, const std::string&) { off_path("save_sdf_multi_octree"); }
void load_sdf_multi_octree(SdfMultiOctree&, const std::string&) { off_path("load_sdf_multi_octree"); }
void save_sdf_augmented_MO(const SdfMultiOctreeAugmented&, const std::string&) { off_path("save_sdf_augmented_MO"); }
void load_sdf_augmented_MO(SdfMultiOctreeAugmented&, const std::string&) { off_path("load_sdf_augmented_MO"); }
void save_sdf_grid(const SdfGridView&, const std::string&) { off_path("save_sdf_grid"); }
void load_sdf_grid(SdfGrid&, const std::string&) { off_path("load_sdf_grid"); }
void save_sdf_frame_octree(const SdfFrameOctreeView&, const std::string&) { off_path("save_sdf_frame_octree"); }
void load_sdf_frame_octree(std::vector<SdfFrameOctreeNode>&, const std::string&) { off_path("load_sdf_frame_octree"); }
void save_sdf_SVS(const SdfSVSView&, const std::string&) { off_path("save_sdf_SVS"); }
void load_sdf_SVS(std::vector<SdfSVSNode>&, const std::string&) { off_path("load_sdf_SVS"); }
void save_sdf_SBS(const SdfSBSView&, const std::filesystem::path&) { off_path("save_sdf_SBS"); }
void load_sdf_SBS(SdfSBS&, const std::filesystem::path&) { off_path("load_sdf_SBS"); }

namespace scom {
void initialize_rot_transforms(std::vector<float4x4>&, int) { off_path("scom::initialize_rot_transforms"); }
void initialize_rot_modifiers(std::vector<int4>&, int) { off_path("scom::initialize_rot_modifiers"); }
} // namespace scom

namespace scom2 {
const Subgroup* create_subgroup(TransformSubgroup, int, int) { off_path("scom2::create_subgroup"); }
} // namespace scom2

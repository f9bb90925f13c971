"""ctypes / numpy mirror of the C-ABI declared in include/lrt_b200.h.

The numpy dtypes reproduce the reference's device-visible structs byte for
byte (CRT_Hit CrossRT/CrossRT.h:26-33, BVHNode/BVHNodePair
utils/raytracing/cbvh.h:21-33, GeomData/InstanceData
utils/raytracing/intersection_common.h:33-56, the SDF nodes of
sdf/simple/sdf_simple_shared.h:23-55 and MultiRenderPreset
core/render_settings.h:116-137).
"""
import ctypes as C

import numpy as np

HIT_DTYPE = np.dtype([("t", "<f4"), ("primId", "<u4"), ("instId", "<u4"), ("geomId", "<u4"),
                      ("coords", "<f4", (4,))])
BVH_NODE_DTYPE = np.dtype([("boxMin", "<f4", (3,)), ("leftOffset", "<u4"), ("boxMax", "<f4", (3,)),
                           ("escapeIndex", "<u4")])
BVH_PAIR_DTYPE = np.dtype([("left", BVH_NODE_DTYPE), ("right", BVH_NODE_DTYPE)])
GEOM_DATA_DTYPE = np.dtype([("boxMin", "<f4", (4,)), ("boxMax", "<f4", (4,)), ("bvhOffset", "<u4"),
                            ("type", "<u4"), ("offset", "<u4", (2,)), ("hasChannels", "<u4"),
                            ("_pad", "<u4", (3,))])
INSTANCE_DTYPE = np.dtype([("boxMin", "<f4", (4,)), ("boxMax", "<f4", (4,)), ("geomId", "<u4"),
                           ("_pad", "<u4", (7,)), ("transform", "<f4", (16,)), ("transformInv", "<f4", (16,)),
                           ("transformInvTransposed", "<f4", (16,))])
FRAME_OCTREE_NODE_DTYPE = np.dtype([("values", "<f4", (8,)), ("offset", "<u4")])
SVS_NODE_DTYPE = np.dtype([("pos_xy", "<u4"), ("pos_z_lod_size", "<u4"), ("values", "<u4", (2,))])
SBS_NODE_DTYPE = np.dtype([("pos_xy", "<u4"), ("pos_z_lod_size", "<u4"), ("data_offset", "<u4"),
                           ("_pad", "<u4")])
SBS_HEADER_DTYPE = np.dtype([("brick_size", "<u4"), ("brick_pad", "<u4"), ("bytes_per_value", "<u4"),
                             ("aux_data", "<u4")])

# Light, core/IRenderer.h:72-78 (lrt_light)
LIGHT_DTYPE = np.dtype([("space", "<f4", (3,)), ("type", "<u4"), ("color", "<f4", (3,)), ("_pad", "<u4")])
LIGHT_DIRECT, LIGHT_POINT, LIGHT_AMBIENT = 0, 1, 2
# MultiRendererMaterial, core/IRenderer.h:31-38 (lrt_material)
MATERIAL_DTYPE = np.dtype([("type", "<u4"), ("texId", "<u4"), ("metallic", "<f4"), ("roughness", "<f4"),
                           ("base_color", "<f4", (4,))])
MATERIAL_COLORED, MATERIAL_TEXTURED = 0, 1
assert MATERIAL_DTYPE.itemsize == 32
# BuildOptions, CrossRT/CrossRT.h:14-17 (LRT_BUILD_*): LOW builds the tree on the device
BUILD_LOW, BUILD_MEDIUM, BUILD_HIGH, BUILD_REFIT = 0x1, 0x2, 0x4, 0x8
assert LIGHT_DTYPE.itemsize == 32
assert HIT_DTYPE.itemsize == 32 and BVH_NODE_DTYPE.itemsize == 32 and BVH_PAIR_DTYPE.itemsize == 64
assert GEOM_DATA_DTYPE.itemsize == 64 and INSTANCE_DTYPE.itemsize == 256
assert FRAME_OCTREE_NODE_DTYPE.itemsize == 36 and SVS_NODE_DTYPE.itemsize == 16
assert SBS_NODE_DTYPE.itemsize == 16 and SBS_HEADER_DTYPE.itemsize == 16

LRT_COUNTER_COUNT = 13
COUNTER_NAMES = ("tlas_nodes", "instances", "blas_pairs", "leaf_calls", "tri_tests", "bricks", "voxels",
                 "st_steps", "octree_leaves", "svs_leaves", "hits", "normals", "voxel_loads")

# Constants (core/render_settings.h, MultiRenderer/BVH2Common.h:30-43, sdf_simple_shared.h:12-20)
TYPE_MESH_TRIANGLE = 0
TYPE_SDF_FRAME_OCTREE = 3
TYPE_SDF_SVS = 5
TYPE_SDF_SBS = 6
TYPE_SDF_SBS_TEX = 10
TYPE_SDF_SBS_COL = 11
TAG_NONE, TAG_TRIANGLE, TAG_SDF_BRICK, TAG_SDF_NODE = 0, 1, 4, 8
SBS_LAYOUT_DX = 1 << 24
SBS_LAYOUT_ID32F_IRGB32F = 4 << 24
INVALID = 0xFFFFFFFF

LRT_TRACE_DEVICE_POINTERS = 0x1
LRT_TRACE_FAST_MATH = 0x2
LRT_TRACE_COUNT_WORK = 0x4
LRT_TRACE_NATURAL_ORDER = 0x8  # image-order and repeated device traces: no longest-first schedule

STATUS_NAMES = {0: "LRT_OK", 1: "LRT_ERR_INVALID_ARGUMENT", 2: "LRT_ERR_BAD_SCENE", 3: "LRT_ERR_NOT_COMMITTED",
                4: "LRT_ERR_CUDA", 5: "LRT_ERR_DEVICE_LIMIT", 6: "LRT_ERR_UNSUPPORTED", 7: "LRT_ERR_OUT_OF_MEMORY"}


class Preset(C.Structure):
    """MultiRenderPreset (core/render_settings.h:116-137)."""
    _fields_ = [("render_mode", C.c_uint32), ("sdf_node_intersect", C.c_uint32), ("normal_mode", C.c_uint32),
                ("ray_gen_mode", C.c_uint32), ("interpolation_mode", C.c_uint32),
                ("representation_mode", C.c_uint32), ("spp", C.c_uint32), ("fixed_lod", C.c_uint32),
                ("level_of_detail", C.c_float), ("compact_sdf_eps", C.c_float), ("LOD_distance", C.c_float),
                ("channel_render_mode", C.c_uint32), ("channel_id", C.c_uint32), ("component_id", C.c_uint32),
                ("CTF_id", C.c_uint32)]


class Camera(C.Structure):
    """lrt_camera: inverse projection / world-view matrices (column-major)."""
    _fields_ = [("proj_inv", C.c_float * 16), ("world_view_inv", C.c_float * 16), ("width", C.c_uint32),
                ("height", C.c_uint32), ("tnear", C.c_float), ("tfar", C.c_float)]


class BatchShape(C.Structure):
    """lrt_batch_shape: launch shape of the batched multi-camera trace."""
    _fields_ = [("tile_w", C.c_uint32), ("tile_h", C.c_uint32), ("rays_per_lane", C.c_uint32),
                ("stack_cap", C.c_uint32)]

    def as_tuple(self):
        return (self.tile_w, self.tile_h, self.rays_per_lane, self.stack_cap)


class TuneEntry(C.Structure):
    _fields_ = [("shape", BatchShape), ("ms", C.c_float)]


LRT_BATCH_NO_GRAPH = 0x1


def default_preset():
    """getDefaultPreset() (core/render_settings.h:139-160)."""
    return Preset(render_mode=1, sdf_node_intersect=1, normal_mode=1, ray_gen_mode=0, interpolation_mode=0,
                  representation_mode=1, spp=1, fixed_lod=1, level_of_detail=16.0, compact_sdf_eps=0.05,
                  LOD_distance=10.0, channel_render_mode=0, channel_id=0, component_id=0, CTF_id=0)


def parity_preset():
    """The preset the hot path is specified for: LAMBERT_NO_TEX, sphere tracing,
    geometric normals, trilinear, volume (the reference default differs in
    sdf_node_intersect=ANALYTIC and normal_mode=VERTEX)."""
    p = default_preset()
    p.sdf_node_intersect = 0
    p.normal_mode = 0
    return p


ARRAY_FIELDS = (
    ("nodesTLAS", BVH_NODE_DTYPE), ("allNodePairs", BVH_PAIR_DTYPE), ("instanceData", INSTANCE_DTYPE),
    ("geomData", GEOM_DATA_DTYPE), ("geomTags", np.dtype("<u4")), ("startEnd", np.dtype(("<u4", (2,)))),
    ("primIdCount", np.dtype("<u4")), ("indices", np.dtype("<u4")), ("vertPos", np.dtype(("<f4", (4,)))),
    ("primIndices", np.dtype("<u4")), ("origNodes", BVH_NODE_DTYPE),
    ("sdfFrameOctreeNodes", FRAME_OCTREE_NODE_DTYPE), ("sdfFrameOctreeRoots", np.dtype("<u4")),
    ("sdfSVSNodes", SVS_NODE_DTYPE), ("sdfSVSRoots", np.dtype("<u4")), ("sdfSBSNodes", SBS_NODE_DTYPE),
    ("sdfSBSData", np.dtype("<u4")), ("sdfSBSDataF", np.dtype("<f4")), ("sdfSBSRoots", np.dtype("<u4")),
    ("sdfSBSHeaders", SBS_HEADER_DTYPE),
)


class SceneArrays(C.Structure):
    """lrt_scene_arrays: {pointer, element count} per BVHRT member."""
    _fields_ = [f for name, _ in ARRAY_FIELDS for f in ((name, C.c_void_p), (name + "_count", C.c_uint64))]


def arrays_to_struct(arrays):
    """dict name -> numpy array  ->  (SceneArrays, keep-alive list)."""
    s = SceneArrays()
    keep = []
    for name, dt in ARRAY_FIELDS:
        a = arrays.get(name)
        if a is None or np.asarray(a).size == 0:
            setattr(s, name, None)
            setattr(s, name + "_count", 0)
            continue
        a = np.ascontiguousarray(a)
        if a.nbytes % dt.itemsize != 0:
            raise ValueError("%s: %d bytes is not a whole number of %d-byte elements" % (name, a.nbytes, dt.itemsize))
        keep.append(a)
        setattr(s, name, a.ctypes.data)
        setattr(s, name + "_count", a.nbytes // dt.itemsize)
    return s, keep


def struct_to_arrays(s):
    """SceneArrays of borrowed pointers -> dict of numpy copies."""
    out = {}
    for name, dt in ARRAY_FIELDS:
        n = getattr(s, name + "_count")
        p = getattr(s, name)
        if not n or not p:
            out[name] = np.zeros(0, dtype=dt)
            continue
        buf = (C.c_char * (n * dt.itemsize)).from_address(p)
        out[name] = np.frombuffer(buf, dtype=dt).copy()
    return out

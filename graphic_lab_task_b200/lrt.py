"""Python host binding of liblrt_b200.so, mirroring the reference's scene API.

``SceneRT`` follows CrossRT's ISceneObject (CrossRT/CrossRT.h:43-175) and the
BVHRT SDF adders (MultiRenderer/BVH2Common.h:95-104): same method names,
argument meaning and call order (AddGeom_* -> AddInstance -> CommitScene ->
RayQuery_NearestHit).  Errors are raised as ``LrtError`` carrying the
library's status and message; nothing falls back to a CPU path — if the CUDA
library is missing or no GPU is present the calls fail loudly.
"""
import ctypes as C
import os

import numpy as np

from ._abi import (HIT_DTYPE, LIGHT_DTYPE, MATERIAL_DTYPE, LRT_BATCH_NO_GRAPH, LRT_COUNTER_COUNT, LRT_TRACE_COUNT_WORK,
                   LRT_TRACE_DEVICE_POINTERS, LRT_TRACE_FAST_MATH, LRT_TRACE_NATURAL_ORDER, STATUS_NAMES, BatchShape, Camera, Preset,
                   SceneArrays, TuneEntry, arrays_to_struct, parity_preset, struct_to_arrays)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblrt_b200.so")

# Every extern "C" symbol declared in include/lrt_b200.h and include/lrt_workloads.h.
EXPORTED = (
    "lrt_scene_create", "lrt_scene_destroy", "lrt_last_error", "lrt_set_preset", "lrt_default_preset",
    "lrt_clear_geom", "lrt_add_geom_triangles3f", "lrt_add_geom_aabb", "lrt_add_geom_sdf_frame_octree",
    "lrt_add_geom_sdf_svs", "lrt_add_geom_sdf_sbs", "lrt_clear_scene", "lrt_add_instance", "lrt_commit_scene",
    "lrt_scene_upload", "lrt_scene_export", "lrt_trace_nearest", "lrt_trace_sync", "lrt_ray_query_nearest_hit",
    "lrt_ray_query_any_hit", "lrt_get_work_counters", "lrt_generate_eye_rays", "lrt_set_voxel_step_limit",
    "lrt_trace_nearest_noalloc", "lrt_batch_create", "lrt_batch_destroy", "lrt_batch_ray_offsets",
    "lrt_batch_update_cameras", "lrt_batch_set_shape", "lrt_batch_get_shape", "lrt_batch_trace", "lrt_batch_sync",
    "lrt_batch_autotune", "lrt_render_lambert", "lrt_adjoint_lambert_sbs", "lrt_sbs_update_values",
    "lrt_generate_bounce_rays", "lrt_generate_bounce_rays_compact", "lrt_render_rgba8", "lrt_trace_nearest_image",
    "lrt_set_materials", "lrt_set_textures", "lrt_set_texcoords", "lrt_fill_gbuffer_transparency", "lrt_render_lambert_image", "lrt_adjoint_lambert_sbs_image",
    "lrt_generate_bounce_rays_sorted",
    "lrt_update_instance", "lrt_add_geom_sdf_frame_octree_file", "lrt_add_geom_sdf_svs_file",
    "lrt_add_geom_sdf_sbs_file", "lrt_batch_render_rgba8",
    "lrt_wl_noisy_sphere", "lrt_wl_spheres", "lrt_wl_sphere_sdf", "lrt_wl_sbs_from_spheres",
    "lrt_wl_frame_octree_from_spheres", "lrt_wl_svs_from_spheres",
)


# Host-buffer traces of PIPE_MIN_RAYS rays or more are staged in chunks
# (csrc/device.cu, pipeline_chunks): sizes ramp PIPE_CHUNK_MIN -> PIPE_CHUNK
# and back down, one trace launch per chunk.
PIPE_MIN_RAYS, PIPE_CHUNK, PIPE_CHUNK_MIN = 262144, 262144, 32768


def _image_size(image_size, n):
    w, h = (int(v) for v in image_size)
    if w * h != n:
        raise ValueError(f"image_size {w} x {h} does not hold {n} rays")
    return w, h


def pipeline_chunks(n):
    """The chunk sizes of a host-buffer trace of n rays (one launch each)."""
    if n < PIPE_MIN_RAYS:
        return [n] if n else []
    up, m = [], PIPE_CHUNK_MIN
    while m < PIPE_CHUNK:
        up.append(m)
        m *= 2
    ramp = sum(up)
    if n <= 2 * ramp:
        return [min(PIPE_CHUNK_MIN, n - o) for o in range(0, n, PIPE_CHUNK_MIN)]
    mid = n - 2 * ramp
    parts = (mid + PIPE_CHUNK - 1) // PIPE_CHUNK
    return up + [mid // parts + (1 if i < mid % parts else 0) for i in range(parts)] + up[::-1]


class LrtError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


_lib = None


def lib():
    """Load liblrt_b200.so (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from .build import build
        build()
    L = C.CDLL(LIB_PATH)
    vp, u32, u64, sz = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t
    P = C.POINTER
    sig = {
        "lrt_scene_create": [C.c_char_p, C.c_char_p, P(vp)],
        "lrt_scene_destroy": [vp],
        "lrt_set_preset": [vp, P(Preset)],
        "lrt_default_preset": [P(Preset)],
        "lrt_clear_geom": [vp],
        "lrt_add_geom_triangles3f": [vp, vp, sz, vp, sz, u32, sz, P(u32)],
        "lrt_add_geom_aabb": [vp, u32, vp, sz, u32, P(u32)],
        "lrt_add_geom_sdf_frame_octree": [vp, vp, sz, P(u32)],
        "lrt_add_geom_sdf_svs": [vp, vp, sz, P(u32)],
        "lrt_add_geom_sdf_sbs": [vp, vp, vp, sz, vp, sz, vp, sz, P(u32)],
        "lrt_clear_scene": [vp],
        "lrt_add_instance": [vp, u32, vp, P(u32)],
        "lrt_commit_scene": [vp, u32],
        "lrt_update_instance": [vp, u32, vp, u32],
        "lrt_add_geom_sdf_frame_octree_file": [vp, C.c_char_p, P(u32)],
        "lrt_add_geom_sdf_svs_file": [vp, C.c_char_p, P(u32)],
        "lrt_add_geom_sdf_sbs_file": [vp, C.c_char_p, P(u32)],
        "lrt_scene_upload": [vp, P(SceneArrays)],
        "lrt_scene_export": [vp, P(SceneArrays)],
        "lrt_trace_nearest": [vp, vp, vp, u64, vp, u32],
        "lrt_trace_nearest_noalloc": [vp, vp, vp, u64, vp, u32],
        "lrt_render_lambert": [vp, vp, u64, vp, vp, vp],
        "lrt_render_rgba8": [vp, vp, vp, u32, vp, vp, vp],
        "lrt_set_materials": [vp, vp, u32, vp, u64, vp, u32],
        "lrt_set_textures": [vp, vp, vp, u32],
        "lrt_set_texcoords": [vp, u32, vp, u64],
        "lrt_fill_gbuffer_transparency": [vp, vp, vp, vp, vp, vp],
        "lrt_trace_nearest_image": [vp, vp, vp, u32, u32, vp, u32],
        "lrt_generate_bounce_rays": [vp, vp, vp, u64, u64, C.c_float, C.c_float, vp, vp],
        "lrt_generate_bounce_rays_compact": [vp, vp, vp, u64, u64, C.c_float, C.c_float, vp, vp, vp, vp],
        "lrt_generate_bounce_rays_sorted": [vp, vp, vp, u64, u64, C.c_float, C.c_float, vp, vp, vp, vp],
        "lrt_adjoint_lambert_sbs": [vp, vp, u64, vp, vp, vp, vp],
        "lrt_render_lambert_image": [vp, vp, u32, u32, vp, vp, vp, u32],
        "lrt_adjoint_lambert_sbs_image": [vp, vp, u32, u32, vp, vp, vp, vp, u32],
        "lrt_sbs_update_values": [vp, vp, u64, vp, u32],
        "lrt_batch_create": [vp, vp, u32, P(vp)],
        "lrt_batch_destroy": [vp],
        "lrt_batch_ray_offsets": [vp, vp],
        "lrt_batch_update_cameras": [vp, vp],
        "lrt_batch_set_shape": [vp, P(BatchShape)],
        "lrt_batch_get_shape": [vp, P(BatchShape)],
        "lrt_batch_trace": [vp, vp, vp, u32],
        "lrt_batch_sync": [vp, vp],
        "lrt_batch_render_rgba8": [vp, vp, u32, vp, vp, vp],
        "lrt_batch_autotune": [vp, vp, vp, u32, vp, u32, P(u32)],
        "lrt_trace_sync": [vp, vp, C.c_int32],
        "lrt_ray_query_nearest_hit": [vp, vp, vp, vp],
        "lrt_ray_query_any_hit": [vp, vp, vp, P(C.c_int32)],
        "lrt_get_work_counters": [vp, vp],
        "lrt_set_voxel_step_limit": [vp, u32],
        "lrt_generate_eye_rays": [vp, vp, vp, vp],
        "lrt_wl_noisy_sphere": [u32, C.c_float, C.c_float, u64, vp, vp, P(u64), P(u64)],
        "lrt_wl_spheres": [u32, C.c_float, C.c_float, C.c_float, u64, vp],
        "lrt_wl_sbs_from_spheres": [vp, u32, u32, u32, u32, vp, vp, vp, vp, P(u64), P(u64), P(u64)],
        "lrt_wl_frame_octree_from_spheres": [vp, u32, u32, vp, P(u64)],
        "lrt_wl_svs_from_spheres": [vp, u32, u32, vp, P(u64)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int32
    L.lrt_last_error.argtypes = [vp]
    L.lrt_last_error.restype = C.c_char_p
    L.lrt_wl_sphere_sdf.argtypes = [vp, u32, C.c_double, C.c_double, C.c_double]
    L.lrt_wl_sphere_sdf.restype = C.c_double
    _lib = L
    return L


def check(status, scene_handle=None):
    if status != 0:
        msg = lib().lrt_last_error(scene_handle)
        raise LrtError(status, msg.decode() if msg else "")


def _ptr(a):
    return a.ctypes.data if a is not None and len(a) else None


class SceneRT:
    """CreateSceneRT("BVH2Common_B200", build_name, layout_name)."""

    def __init__(self, build_name="cbvh_embree2", layout_name="SuperTreeletAlignedMerged4", preset=None):
        L = lib()
        h = C.c_void_p()
        check(L.lrt_scene_create(build_name.encode() if build_name else None,
                                 layout_name.encode() if layout_name else None, C.byref(h)))
        self.h = h
        self.SetPreset(preset if preset is not None else parity_preset())

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            lib().lrt_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st):
        check(st, self.h)

    # -- ISceneObject ------------------------------------------------------
    def SetPreset(self, preset):
        self.preset = preset
        self._check(lib().lrt_set_preset(self.h, C.byref(preset)))

    def GetPreset(self):
        return self.preset

    def ClearGeom(self):
        self._check(lib().lrt_clear_geom(self.h))

    def AddGeom_Triangles3f(self, vpos3f, tri_indices, flags=4, vByteStride=12):
        v = np.ascontiguousarray(vpos3f, dtype=np.float32).reshape(-1)
        t = np.ascontiguousarray(tri_indices, dtype=np.uint32).reshape(-1)
        nvert = len(v) * 4 // vByteStride
        gid = C.c_uint32()
        self._check(lib().lrt_add_geom_triangles3f(self.h, _ptr(v), nvert, _ptr(t), len(t), flags, vByteStride,
                                                   C.byref(gid)))
        return gid.value

    def AddGeom_AABB(self, typeId, boxMinMaxF8, flags=4):
        b = np.ascontiguousarray(boxMinMaxF8, dtype=np.float32).reshape(-1, 8)
        gid = C.c_uint32()
        self._check(lib().lrt_add_geom_aabb(self.h, typeId, _ptr(b), len(b), flags, C.byref(gid)))
        return gid.value

    def AddGeom_SdfFrameOctree(self, nodes):
        gid = C.c_uint32()
        self._check(lib().lrt_add_geom_sdf_frame_octree(self.h, _ptr(nodes), len(nodes), C.byref(gid)))
        return gid.value

    def AddGeom_SdfSVS(self, nodes):
        gid = C.c_uint32()
        self._check(lib().lrt_add_geom_sdf_svs(self.h, _ptr(nodes), len(nodes), C.byref(gid)))
        return gid.value

    def AddGeom_SdfSBS(self, header, nodes, values, values_f=None):
        hdr = np.ascontiguousarray(header)
        vals = np.ascontiguousarray(values, dtype=np.uint32)
        vf = None if values_f is None else np.ascontiguousarray(values_f, dtype=np.float32)
        gid = C.c_uint32()
        self._check(lib().lrt_add_geom_sdf_sbs(self.h, hdr.ctypes.data, _ptr(nodes), len(nodes), _ptr(vals),
                                               len(vals), _ptr(vf), 0 if vf is None else len(vf), C.byref(gid)))
        return gid.value

    def ClearScene(self):
        self._check(lib().lrt_clear_scene(self.h))

    def AddInstance(self, geomId, matrix_col_major):
        m = np.ascontiguousarray(matrix_col_major, dtype=np.float32).reshape(16)
        iid = C.c_uint32()
        self._check(lib().lrt_add_instance(self.h, geomId, m.ctypes.data, C.byref(iid)))
        return iid.value

    def AddGeom_SdfFile(self, kind, path):
        """Adds an SDF model from a file in the reference's format; kind is
        "frame_octree", "svs" or "sbs".  Returns the geometry id."""
        fn = {"frame_octree": lib().lrt_add_geom_sdf_frame_octree_file, "svs": lib().lrt_add_geom_sdf_svs_file,
              "sbs": lib().lrt_add_geom_sdf_sbs_file}[kind]
        g = C.c_uint32()
        self._check(fn(self.h, os.fsencode(path), C.byref(g)))
        return g.value

    def UpdateInstance(self, inst_id, matrix_col_major, update_normal_matrix=False):
        """ISceneObject::UpdateInstance: takes effect at the next CommitScene."""
        m = np.ascontiguousarray(matrix_col_major, dtype=np.float32).reshape(16)
        self._check(lib().lrt_update_instance(self.h, inst_id, m.ctypes.data, 1 if update_normal_matrix else 0))

    def CommitScene(self, options=4, host_only=False):
        """Builds the TLAS and uploads to the current CUDA device; with
        host_only the arrays are built and validated but not uploaded."""
        self._check(lib().lrt_commit_scene(self.h, options | (0x100 if host_only else 0)))

    def RayQuery_NearestHit(self, posAndNear, dirAndFar):
        pn = np.ascontiguousarray(posAndNear, dtype=np.float32)
        df = np.ascontiguousarray(dirAndFar, dtype=np.float32)
        hit = np.zeros(1, dtype=HIT_DTYPE)
        self._check(lib().lrt_ray_query_nearest_hit(self.h, pn.ctypes.data, df.ctypes.data, hit.ctypes.data))
        return hit[0]

    def RayQuery_AnyHit(self, posAndNear, dirAndFar):
        pn = np.ascontiguousarray(posAndNear, dtype=np.float32)
        df = np.ascontiguousarray(dirAndFar, dtype=np.float32)
        out = C.c_int32()
        self._check(lib().lrt_ray_query_any_hit(self.h, pn.ctypes.data, df.ctypes.data, C.byref(out)))
        return bool(out.value)

    # -- batched form and the drop-in array boundary -----------------------
    def RayQuery_NearestHitBatch(self, rays, fast_math=False, count_work=False):
        """rays: (n, 8) float32 host array {posAndNear, dirAndFar} -> hits (n,) HIT_DTYPE."""
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        hits = np.zeros(len(r), dtype=HIT_DTYPE)
        flags = (LRT_TRACE_FAST_MATH if fast_math else 0) | (LRT_TRACE_COUNT_WORK if count_work else 0)
        self._check(lib().lrt_trace_nearest(self.h, r.ctypes.data, hits.ctypes.data, len(r), None, flags))
        return hits

    def trace_host(self, rays_ptr, hits_ptr, n, fast_math=False):
        """Synchronous trace of host buffers, staged through device memory:
        from PIPE_MIN_RAYS rays on in a chunked copy/trace/copy pipeline
        (page-locked buffers let both copy directions overlap)."""
        flags = LRT_TRACE_FAST_MATH if fast_math else 0
        self._check(lib().lrt_trace_nearest(self.h, C.c_void_p(rays_ptr), C.c_void_p(hits_ptr), n, None, flags))

    def trace_device(self, rays_ptr, hits_ptr, n, stream=0, fast_math=False, count_work=False, natural_order=False):
        """Asynchronous trace of device buffers (16-byte aligned) on `stream`;
        natural_order: no schedule for the 32-ray groups of a large trace."""
        flags = LRT_TRACE_DEVICE_POINTERS | (LRT_TRACE_FAST_MATH if fast_math else 0) | \
            (LRT_TRACE_COUNT_WORK if count_work else 0) | (LRT_TRACE_NATURAL_ORDER if natural_order else 0)
        self._check(lib().lrt_trace_nearest(self.h, C.c_void_p(rays_ptr), C.c_void_p(hits_ptr), n,
                                            C.c_void_p(stream) if stream else None, flags))

    def trace_image(self, rays_ptr, hits_ptr, width, height, stream=0, fast_math=False, count_work=False,
                    natural_order=False):
        """Asynchronous trace of the device rays of a width x height image
        (row-major pixels), in 8x4-pixel tiles per warp, the stream's
        longest-first tile schedule unless natural_order."""
        flags = (LRT_TRACE_FAST_MATH if fast_math else 0) | (LRT_TRACE_COUNT_WORK if count_work else 0) | \
            (LRT_TRACE_NATURAL_ORDER if natural_order else 0)
        self._check(lib().lrt_trace_nearest_image(self.h, C.c_void_p(rays_ptr), C.c_void_p(hits_ptr), width, height,
                                                  C.c_void_p(stream) if stream else None, flags))

    def sync(self, stream=0, read_counters=False):
        self._check(lib().lrt_trace_sync(self.h, C.c_void_p(stream) if stream else None, int(read_counters)))

    def generate_bounce_rays(self, rays_ptr, hits_ptr, n, seed, out_ptr, tnear=1e-4, tfar=1e9, stream=0):
        self._check(lib().lrt_generate_bounce_rays(self.h, C.c_void_p(rays_ptr), C.c_void_p(hits_ptr), n, seed,
                                                   tnear, tfar, C.c_void_p(out_ptr),
                                                   C.c_void_p(stream) if stream else None))

    # -- differentiable form (SBS distances) ------------------------------
    def generate_bounce_rays_compact(self, rays_ptr, hits_ptr, n, seed, out_ptr, index_ptr, count_ptr, tnear=1e-4,
                                     tfar=1e9, stream=0):
        """Bounce rays of the hits only, in ray order; index_ptr (uint32) maps
        them to the traced rays, count_ptr (device uint64) receives their number."""
        self._check(lib().lrt_generate_bounce_rays_compact(self.h, C.c_void_p(rays_ptr), C.c_void_p(hits_ptr), n,
                                                           seed, tnear, tfar, C.c_void_p(out_ptr),
                                                           C.c_void_p(index_ptr), C.c_void_p(count_ptr),
                                                           C.c_void_p(stream) if stream else None))

    def generate_bounce_rays_sorted(self, rays_ptr, hits_ptr, n, seed, out_ptr, index_ptr, count_ptr, tnear=1e-4,
                                    tfar=1e9, stream=0):
        """generate_bounce_rays_compact in coherence order (direction cell,
        then the origin's Morton code in the scene box); index_ptr (uint32, n
        entries) maps them to the traced rays."""
        self._check(lib().lrt_generate_bounce_rays_sorted(self.h, C.c_void_p(rays_ptr), C.c_void_p(hits_ptr), n,
                                                          seed, tnear, tfar, C.c_void_p(out_ptr),
                                                          C.c_void_p(index_ptr), C.c_void_p(count_ptr),
                                                          C.c_void_p(stream) if stream else None))

    def render_lambert(self, rays_ptr, n, light, image_ptr, stream=0, image_size=None, natural_order=False):
        """Lambert image of n device rays.  image_size=(width, height) with
        width * height == n: the rays are an image (views stacked as rows),
        traced in 8x4-pixel tiles in the stream's tile schedule unless
        natural_order."""
        L = (C.c_float * 3)(*[float(x) for x in light])
        st = C.c_void_p(stream) if stream else None
        if image_size is None:
            self._check(lib().lrt_render_lambert(self.h, C.c_void_p(rays_ptr), n, L, C.c_void_p(image_ptr), st))
            return
        w, h = _image_size(image_size, n)
        self._check(lib().lrt_render_lambert_image(self.h, C.c_void_p(rays_ptr), w, h, L, C.c_void_p(image_ptr), st,
                                                   LRT_TRACE_NATURAL_ORDER if natural_order else 0))

    def render_rgba8(self, camera, lights, background, image_ptr, stream=0):
        """Fused Render (eye rays, nearest hit, LAMBERT_NO_TEX resolve with
        `lights` — a LIGHT_DTYPE array —, tonemap) of `camera` into
        width*height RGBA8 pixels of device memory."""
        lt = np.ascontiguousarray(lights, dtype=LIGHT_DTYPE)
        bg = (C.c_float * 4)(*[float(x) for x in background])
        self._check(lib().lrt_render_rgba8(self.h, C.byref(camera), lt.ctypes.data if len(lt) else None, len(lt), bg,
                                           C.c_void_p(image_ptr), C.c_void_p(stream) if stream else None))

    def set_materials(self, materials, mat_id_by_prim_id, mat_id_offsets):
        """MultiRenderer's m_materials (MATERIAL_DTYPE), m_matIdbyPrimId and
        m_matIdOffsets ({start, size} per geometry), copied."""
        m = np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)
        ids = np.ascontiguousarray(mat_id_by_prim_id, dtype=np.uint32).reshape(-1)
        offs = np.ascontiguousarray(mat_id_offsets, dtype=np.uint32).reshape(-1)
        self._check(lib().lrt_set_materials(self.h, m.ctypes.data if len(m) else None, len(m),
                                            ids.ctypes.data if len(ids) else None, len(ids),
                                            offs.ctypes.data if len(offs) else None, len(offs) // 2))

    def set_textures(self, images):
        """MultiRenderer's m_textures: a list of (h, w, 4) float32 images
        (slot k = images[k]), sampled bilinear with clamped addressing."""
        imgs = [np.ascontiguousarray(i, np.float32) for i in (images or [])]
        dims = np.array([[i.shape[1], i.shape[0]] for i in imgs], np.uint32).reshape(-1)
        texels = np.concatenate([i.reshape(-1) for i in imgs]) if imgs else np.zeros(0, np.float32)
        self._check(lib().lrt_set_textures(self.h, texels.ctypes.data if len(texels) else None,
                                           dims.ctypes.data if len(dims) else None, len(imgs)))

    def set_texcoords(self, geom_id, texcoords):
        """Per-vertex texture coordinates (nverts, 2) of triangle geometry geom_id (None clears them)."""
        if texcoords is None:
            self._check(lib().lrt_set_texcoords(self.h, geom_id, None, 0))
            return
        tc = np.ascontiguousarray(texcoords, np.float32).reshape(-1, 2)
        self._check(lib().lrt_set_texcoords(self.h, geom_id, tc.ctypes.data, len(tc)))

    def fill_gbuffer_transparency(self, camera, background, transparency_ptr, hits_ptr, stream=0):
        """kernel1D_FillGbufferWithTransparency for `camera`: float4
        {rgb, alpha} and the last hit per pixel, in device memory."""
        bg = (C.c_float * 4)(*[float(x) for x in background])
        self._check(lib().lrt_fill_gbuffer_transparency(self.h, C.byref(camera), bg, C.c_void_p(transparency_ptr),
                                                        C.c_void_p(hits_ptr), C.c_void_p(stream) if stream else None))

    def adjoint_lambert(self, rays_ptr, n, light, dimage_ptr, grad_ptr, stream=0, image_size=None,
                        natural_order=False):
        """Adds dLoss/d(SBS float values) of the Lambert image of n device
        rays to grad_ptr; image_size and natural_order as render_lambert."""
        L = (C.c_float * 3)(*[float(x) for x in light])
        st = C.c_void_p(stream) if stream else None
        if image_size is None:
            self._check(lib().lrt_adjoint_lambert_sbs(self.h, C.c_void_p(rays_ptr), n, L, C.c_void_p(dimage_ptr),
                                                      C.c_void_p(grad_ptr), st))
            return
        w, h = _image_size(image_size, n)
        self._check(lib().lrt_adjoint_lambert_sbs_image(self.h, C.c_void_p(rays_ptr), w, h, L, C.c_void_p(dimage_ptr),
                                                        C.c_void_p(grad_ptr), st,
                                                        LRT_TRACE_NATURAL_ORDER if natural_order else 0))

    def update_sbs_values(self, values_ptr, count, device=True, stream=0):
        self._check(lib().lrt_sbs_update_values(self.h, C.c_void_p(values_ptr), count,
                                                C.c_void_p(stream) if stream else None,
                                                LRT_TRACE_DEVICE_POINTERS if device else 0))

    def set_voxel_step_limit(self, steps):
        self._check(lib().lrt_set_voxel_step_limit(self.h, steps))

    def work_counters(self):
        c = np.zeros(LRT_COUNTER_COUNT, dtype=np.uint64)
        self._check(lib().lrt_get_work_counters(self.h, c.ctypes.data))
        return c

    def upload_arrays(self, arrays):
        s, keep = arrays_to_struct(arrays)
        self._check(lib().lrt_scene_upload(self.h, C.byref(s)))
        del keep

    def export_arrays(self):
        s = SceneArrays()
        self._check(lib().lrt_scene_export(self.h, C.byref(s)))
        return struct_to_arrays(s)

    def generate_eye_rays(self, camera, rays_ptr, stream=0):
        self._check(lib().lrt_generate_eye_rays(self.h, C.byref(camera), C.c_void_p(rays_ptr),
                                                C.c_void_p(stream) if stream else None))


class CameraBatch:
    """Batched multi-camera trace over a committed SceneRT (lrt_batch_*):
    one persistent launch for all cameras, replayed from a CUDA graph."""

    def __init__(self, scene, cameras):
        self.scene = scene
        self.n = len(cameras)
        arr = (Camera * self.n)(*cameras)
        h = C.c_void_p()
        scene._check(lib().lrt_batch_create(scene.h, arr, self.n, C.byref(h)))
        self.h = h
        off = np.zeros(self.n + 1, np.uint64)
        scene._check(lib().lrt_batch_ray_offsets(self.h, off.ctypes.data))
        self.offsets = off
        self.total_rays = int(off[-1])

    def close(self):
        if getattr(self, "h", None):
            lib().lrt_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def update_cameras(self, cameras):
        arr = (Camera * self.n)(*cameras)
        self.scene._check(lib().lrt_batch_update_cameras(self.h, arr))

    @property
    def shape(self):
        s = BatchShape()
        self.scene._check(lib().lrt_batch_get_shape(self.h, C.byref(s)))
        return s.as_tuple()

    def set_shape(self, tile_w, tile_h, rays_per_lane, stack_cap):
        s = BatchShape(tile_w, tile_h, rays_per_lane, stack_cap)
        self.scene._check(lib().lrt_batch_set_shape(self.h, C.byref(s)))

    def trace(self, hits_ptr, stream=0, graph=True):
        self.scene._check(lib().lrt_batch_trace(self.h, C.c_void_p(hits_ptr), C.c_void_p(stream) if stream else None,
                                                0 if graph else LRT_BATCH_NO_GRAPH))

    def render_rgba8(self, lights, background, images_ptr, stream=0):
        """All cameras' RGBA8 images in one launch (offsets as the rays')."""
        lt = np.ascontiguousarray(lights, dtype=LIGHT_DTYPE)
        bg = (C.c_float * 4)(*[float(x) for x in background])
        self.scene._check(lib().lrt_batch_render_rgba8(self.h, lt.ctypes.data if len(lt) else None, len(lt), bg,
                                                       C.c_void_p(images_ptr), C.c_void_p(stream) if stream else None))

    def sync(self, stream=0):
        self.scene._check(lib().lrt_batch_sync(self.h, C.c_void_p(stream) if stream else None))

    def autotune(self, hits_ptr, stream=0, reps=3):
        table = (TuneEntry * 64)()
        n = C.c_uint32()
        self.scene._check(lib().lrt_batch_autotune(self.h, C.c_void_p(hits_ptr), C.c_void_p(stream) if stream else None,
                                                   reps, table, 64, C.byref(n)))
        return [(table[i].shape.as_tuple(), float(table[i].ms)) for i in range(n.value)]

"""Python bindings of the checkers (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Two checkers:

* ``Port`` — oracle/lrt_oracle.c, the C restatement of the reference ray query,
  built into oracle/_build/liblrt_oracle.so.
* ``RefScene`` — the reference's own BVHRT compiled from its sources
  (oracle/_ref/liblrt_ref.so, bit-parity build; liblrt_ref_fast.so, the
  reference's Release flags), driven through oracle/ref/ref_harness.cpp.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from graphic_lab_task_b200._abi import (HIT_DTYPE, LRT_COUNTER_COUNT, Preset, SceneArrays, arrays_to_struct,
                                        parity_preset, struct_to_arrays)

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "liblrt_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "liblrt_ref.so")
REF_FAST_SO = os.path.join(HERE, "_ref", "liblrt_ref_fast.so")
DROPIN_SO = os.path.join(HERE, "_ref", "liblrt_b200_dropin.so")
WL_SO = os.path.join(HERE, "_build", "liblrt_workloads.so")


def reference_src():
    """The reference checkout the checker build compiles from: the
    LRT_REFERENCE environment variable, else oracle/Makefile's default."""
    r = subprocess.run(["make", "-s", "-C", HERE, "ref-path"], capture_output=True, text=True)
    return r.stdout.strip() if r.returncode == 0 else ""


def build(with_reference=True):
    """Compile the C restatement, the seeded-workload library of the bench's
    reference arm and, where the reference sources exist, the reference
    build (oracle/Makefile)."""
    targets = ["port", "wl"]
    src = reference_src() if with_reference else ""
    if src and os.path.isdir(src):
        targets += ["ref", "dropin"]
    subprocess.run(["make", "-s", "-C", HERE, "-j8"] + targets, check=True)


_port = None
_refs = {}


def port_lib():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            build(with_reference=False)
        lib = C.CDLL(PORT_SO)
        lib.lrto_trace.restype = C.c_uint64
        lib.lrto_trace.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_void_p, C.c_uint64,
                                   C.c_void_p, C.c_int]
        lib.lrto_trace_counted.restype = None
        lib.lrto_trace_counted.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_void_p,
                                           C.c_uint64, C.c_void_p]
        _port = lib
    return _port


def ref_available(fast=False):
    return os.path.exists(REF_FAST_SO if fast else REF_SO)


def dropin_available():
    return os.path.exists(DROPIN_SO)


def ref_lib(fast=False, dropin=False):
    key = "dropin" if dropin else bool(fast)
    if key not in _refs:
        path = DROPIN_SO if dropin else (REF_FAST_SO if fast else REF_SO)
        if not os.path.exists(path):
            raise RuntimeError("reference build %s is missing (make -C oracle ref)" % path)
        lib = C.CDLL(path)
        lib.lrtr_create.restype = C.c_void_p
        lib.lrtr_create.argtypes = [C.c_char_p, C.c_char_p]
        lib.lrtr_destroy.argtypes = [C.c_void_p]
        lib.lrtr_set_preset.argtypes = [C.c_void_p, C.POINTER(Preset)]
        for fn in ("lrtr_add_triangles", "lrtr_add_frame_octree", "lrtr_add_svs", "lrtr_add_sbs",
                   "lrtr_add_instance"):
            getattr(lib, fn).restype = C.c_uint32
        lib.lrtr_add_triangles.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64]
        lib.lrtr_add_frame_octree.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        lib.lrtr_add_svs.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64]
        lib.lrtr_add_sbs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64,
                                     C.c_void_p, C.c_uint64]
        lib.lrtr_add_instance.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        lib.lrtr_update_instance.restype = None
        lib.lrtr_update_instance.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
        lib.lrtr_commit.argtypes = [C.c_void_p]
        lib.lrtr_export.argtypes = [C.c_void_p, C.POINTER(SceneArrays)]
        lib.lrtr_import.argtypes = [C.c_void_p, C.POINTER(SceneArrays)]
        lib.lrtr_trace.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_int]
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        if dropin:
            lib.lrtd_create.restype = vp
            lib.lrtd_create.argtypes = [C.c_char_p, C.c_char_p]
            lib.lrtd_commit_status.restype = C.c_int32
            lib.lrtd_commit_status.argtypes = [vp, C.c_char_p, u64]
            lib.lrtd_trace_batch.restype = C.c_int32
            lib.lrtd_trace_batch.argtypes = [vp, vp, vp, u64]
        lib.lrtr_renderer_create.restype = vp
        for fn, args in (("lrtr_renderer_create", [vp]), ("lrtr_renderer_destroy", [vp]),
                         ("lrtr_renderer_add_mesh", [vp, u32, vp, u64, vp, u64, vp]),
                         ("lrtr_renderer_add_texture", [vp, u32, u32, vp]),
                         ("lrtr_renderer_set_preset", [vp, C.POINTER(Preset)]),
                         ("lrtr_renderer_set_camera_inverse", [vp, vp, vp]),
                         ("lrtr_renderer_look_at", [vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float]),
                         ("lrtr_renderer_set_lights", [vp, vp, u32]), ("lrtr_renderer_set_background", [vp, vp]),
                         ("lrtr_renderer_set_materials", [vp, vp, u32, vp, u64, vp, u32]),
                         ("lrtr_renderer_set_frame", [vp, u32]), ("lrtr_renderer_eye_rays", [vp, u32, u32, u32, vp]),
                         ("lrtr_renderer_render", [vp, u32, u32, vp]),
                         ("lrtr_renderer_fill_transparency", [vp, u32, u32, u32, vp, vp])):
            if not hasattr(lib, fn):  # a checker library built before the entry point existed
                continue
            getattr(lib, fn).argtypes = args
            if fn not in ("lrtr_renderer_create", "lrtr_renderer_add_texture"):
                getattr(lib, fn).restype = None
        if hasattr(lib, "lrtr_renderer_add_texture"):
            lib.lrtr_renderer_add_texture.restype = u32
        _refs[key] = lib
    return _refs[key]


def port_trace(arrays, rays, preset=None, threads=os.cpu_count(), counters=False):
    """Trace with the C restatement.  Returns hits (and summed counters)."""
    lib = port_lib()
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    hits = np.zeros(len(rays), dtype=HIT_DTYPE)
    cnt = np.zeros(LRT_COUNTER_COUNT, dtype=np.uint64)
    limits = lib.lrto_trace(C.byref(s), C.byref(p), rays.ctypes.data, hits.ctypes.data, len(rays),
                            cnt.ctypes.data, int(threads))
    del keep
    if counters:
        return hits, cnt, int(limits)
    return hits


def port_trace_per_ray_counters(arrays, rays, preset=None):
    lib = port_lib()
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    hits = np.zeros(len(rays), dtype=HIT_DTYPE)
    cnt = np.zeros((len(rays), LRT_COUNTER_COUNT), dtype=np.uint64)
    lib.lrto_trace_counted(C.byref(s), C.byref(p), rays.ctypes.data, hits.ctypes.data, len(rays), cnt.ctypes.data)
    del keep
    return hits, cnt


class RefScene:
    """A reference BVHRT (CreateSceneRT("BVH2Common", ...)) in oracle/_ref."""

    def __init__(self, build_name="cbvh_embree2", layout_name="SuperTreeletAlignedMerged4", fast=False,
                 preset=None):
        self.lib = ref_lib(fast)
        self.h = self.lib.lrtr_create(build_name.encode(), layout_name.encode())
        if not self.h:
            raise RuntimeError("CreateSceneRT failed")
        self.set_preset(preset if preset is not None else parity_preset())

    def close(self):
        if self.h:
            self.lib.lrtr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_preset(self, preset):
        self.preset = preset
        self.lib.lrtr_set_preset(self.h, C.byref(preset))

    def add_triangles(self, verts, tris):
        v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1)
        return self.lib.lrtr_add_triangles(self.h, v.ctypes.data, len(v), t.ctypes.data, len(t))

    def add_frame_octree(self, nodes):
        return self.lib.lrtr_add_frame_octree(self.h, nodes.ctypes.data, len(nodes))

    def add_svs(self, nodes):
        return self.lib.lrtr_add_svs(self.h, nodes.ctypes.data, len(nodes))

    def add_sbs(self, header, nodes, values, values_f=None):
        hdr = np.ascontiguousarray(header)
        vf = np.zeros(0, np.float32) if values_f is None else np.ascontiguousarray(values_f, np.float32)
        vals = np.ascontiguousarray(values, np.uint32)
        return self.lib.lrtr_add_sbs(self.h, hdr.ctypes.data, nodes.ctypes.data, len(nodes), vals.ctypes.data,
                                     len(vals), vf.ctypes.data if len(vf) else None, len(vf))

    def add_instance(self, geom_id, matrix_col_major):
        m = np.ascontiguousarray(matrix_col_major, dtype=np.float32).reshape(16)
        return self.lib.lrtr_add_instance(self.h, geom_id, m.ctypes.data)

    def update_instance(self, inst_id, matrix_col_major):
        m = np.ascontiguousarray(matrix_col_major, dtype=np.float32).reshape(16)
        self.lib.lrtr_update_instance(self.h, inst_id, m.ctypes.data)

    def commit(self):
        self.lib.lrtr_commit(self.h)

    def export(self):
        s = SceneArrays()
        self.lib.lrtr_export(self.h, C.byref(s))
        return struct_to_arrays(s)

    def import_arrays(self, arrays):
        s, keep = arrays_to_struct(arrays)
        self.lib.lrtr_import(self.h, C.byref(s))
        del keep

    def trace(self, rays, threads=1):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        hits = np.zeros(len(rays), dtype=HIT_DTYPE)
        self.lib.lrtr_trace(self.h, rays.ctypes.data, hits.ctypes.data, len(rays), int(threads))
        return hits


class RefRenderer:
    """The reference's own MultiRenderer (MultiRenderer/MultiRenderer*.cpp,
    compiled in oracle/_ref) tracing a RefScene: initEyeRay, Render (fill
    G-buffer, resolve, tonemap) and the transparency AnyHit loop.  Image
    sizes must be multiples of 8 (the renderer's tile padding)."""

    def __init__(self, scene):
        self.scene = scene  # keeps the BVHRT alive
        self.lib = scene.lib
        self.h = self.lib.lrtr_renderer_create(scene.h)

    def close(self):
        if self.h:
            self.lib.lrtr_renderer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_mesh(self, geom_id, verts, tris, texcoords=None):
        """MultiRenderer::add_mesh_internal: the mesh copy the resolve reads
        triangle normals and texture coordinates from (no vertex normals)."""
        v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(tris, np.uint32).reshape(-1)
        tc = None if texcoords is None else np.ascontiguousarray(texcoords, np.float32).reshape(-1, 2)
        assert tc is None or len(tc) == len(v)
        self.lib.lrtr_renderer_add_mesh(self.h, geom_id, v.ctypes.data, len(v), t.ctypes.data, len(t),
                                        tc.ctypes.data if tc is not None else None)

    def add_texture(self, image):
        """MultiRenderer::AddTexture of an (h, w, 4) float32 image; returns its slot (1, 2, ...: every
        slot of a new renderer holds a 16x16 (0, 1, 1, 1) image, slot 0 keeps it)."""
        img = np.ascontiguousarray(image, np.float32)
        return self.lib.lrtr_renderer_add_texture(self.h, img.shape[1], img.shape[0], img.ctypes.data)

    def set_preset(self, preset):
        self.lib.lrtr_renderer_set_preset(self.h, C.byref(preset))

    def set_camera(self, cam):
        """The camera's inverse matrices (lrt_camera.proj_inv, world_view_inv)."""
        p = np.array(cam.proj_inv[:], np.float32)
        w = np.array(cam.world_view_inv[:], np.float32)
        self.lib.lrtr_renderer_set_camera_inverse(self.h, p.ctypes.data, w.ctypes.data)

    def look_at(self, eye, center, up, fovy, aspect, znear=0.01, zfar=100.0):
        """LiteMath lookAt / perspectiveMatrix + MultiRenderer::UpdateCamera."""
        e, c, u = (np.ascontiguousarray(x, np.float32) for x in (eye, center, up))
        self.lib.lrtr_renderer_look_at(self.h, e.ctypes.data, c.ctypes.data, u.ctypes.data, fovy, aspect, znear, zfar)

    def set_lights(self, lights):
        from graphic_lab_task_b200._abi import LIGHT_DTYPE
        lt = np.ascontiguousarray(lights, dtype=LIGHT_DTYPE)
        self.lib.lrtr_renderer_set_lights(self.h, lt.ctypes.data if len(lt) else None, len(lt))

    def set_background(self, rgba):
        bg = np.ascontiguousarray(rgba, np.float32)
        self.lib.lrtr_renderer_set_background(self.h, bg.ctypes.data)

    def set_materials(self, materials, mat_ids, mat_offsets):
        from graphic_lab_task_b200._abi import MATERIAL_DTYPE
        m = np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)
        ids = np.ascontiguousarray(mat_ids, np.uint32)
        offs = np.ascontiguousarray(mat_offsets, np.uint32).reshape(-1)
        self.lib.lrtr_renderer_set_materials(self.h, m.ctypes.data, len(m), ids.ctypes.data, len(ids),
                                             offs.ctypes.data, len(offs) // 2)

    def set_frame(self, frame):
        self.lib.lrtr_renderer_set_frame(self.h, frame)

    def eye_rays(self, width, height, sample=0):
        out = np.zeros((width * height, 8), np.float32)
        self.lib.lrtr_renderer_eye_rays(self.h, width, height, sample, out.ctypes.data)
        return out

    def render(self, width, height):
        img = np.zeros(width * height, np.uint32)
        self.lib.lrtr_renderer_render(self.h, width, height, img.ctypes.data)
        return img

    def fill_transparency(self, width, height, sample=0):
        transp = np.zeros((width * height, 4), np.float32)
        gb = np.zeros(width * height, HIT_DTYPE)
        self.lib.lrtr_renderer_fill_transparency(self.h, width, height, sample, transp.ctypes.data, gb.ctypes.data)
        return transp, gb


class DropInScene(RefScene):
    """The reference's BVHRT with the BVHRT_B200 subclass of INTEGRATION.md
    (oracle/ref/bvhrt_b200.cpp, linked against liblrt_b200.so): the
    reference's own adders and CommitScene build the scene, the override
    uploads it, and ray queries run on the GPU.  `trace` goes through the
    virtual RayQuery_NearestHit one ray at a time (threads=1); `trace_batch`
    through RayQuery_NearestHitBatch."""

    def __init__(self, build_name="cbvh_embree2", layout_name="SuperTreeletAlignedMerged4", preset=None):
        self.lib = ref_lib(dropin=True)
        self.h = self.lib.lrtd_create(build_name.encode(), layout_name.encode())
        if not self.h:
            raise RuntimeError("BVHRT_B200: lrt_scene_create failed")
        self.set_preset(preset if preset is not None else parity_preset())

    def commit(self):
        self.lib.lrtr_commit(self.h)
        msg = C.create_string_buffer(512)
        st = self.lib.lrtd_commit_status(self.h, msg, len(msg))
        if st != 0:
            raise RuntimeError("BVHRT_B200::CommitScene upload failed (%d): %s" % (st, msg.value.decode()))

    def trace_batch(self, rays):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
        hits = np.zeros(len(rays), dtype=HIT_DTYPE)
        st = self.lib.lrtd_trace_batch(self.h, rays.ctypes.data, hits.ctypes.data, len(rays))
        if st != 0:
            raise RuntimeError("RayQuery_NearestHitBatch failed with status %d" % st)
        return hits


_port_textures = None


def port_set_textures(images, vert_tc=None):
    """The textures (a list of (h, w, 4) float32 images, slot k = images[k])
    and the per-vertex texture coordinates ((nverts, 2), parallel to the
    scene's vertPos; None: zeros) of the restated renderer's next calls."""
    global _port_textures
    lib = port_lib()
    if not hasattr(lib, "_tex_bound"):
        lib.lrto_set_textures.restype = None
        lib.lrto_set_textures.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64]
        lib._tex_bound = True
    imgs = [np.ascontiguousarray(i, np.float32) for i in (images or [])]
    dims = np.array([[i.shape[1], i.shape[0]] for i in imgs], np.uint32).reshape(-1)
    offs = np.cumsum([0] + [i.shape[0] * i.shape[1] for i in imgs])[:-1].astype(np.uint64)
    texels = np.concatenate([i.reshape(-1) for i in imgs]) if imgs else np.zeros(4, np.float32)
    tc = None if vert_tc is None else np.ascontiguousarray(vert_tc, np.float32).reshape(-1, 2)
    _port_textures = (texels, dims, offs, tc)  # kept alive for the C side
    lib.lrto_set_textures(texels.ctypes.data, dims.ctypes.data if len(dims) else None,
                          offs.ctypes.data if len(offs) else None, len(imgs),
                          tc.ctypes.data if tc is not None else None, 0 if tc is None else len(tc))


def port_render_lambert(arrays, rays, light, preset=None, threads=os.cpu_count()):
    """Float Lambert image of the rays (the restatement of the GPU forward)."""
    lib = port_lib()
    if not hasattr(lib, "_render_bound"):
        lib.lrto_render_lambert.restype = None
        lib.lrto_render_lambert.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_uint64,
                                            C.c_void_p, C.c_void_p, C.c_int]
        lib.lrto_adjoint_lambert_fp64.restype = None
        lib.lrto_adjoint_lambert_fp64.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_uint64,
                                                  C.c_void_p, C.c_void_p, C.c_void_p]
        lib._render_bound = True
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    L = np.ascontiguousarray(light, dtype=np.float32)
    img = np.zeros(len(rays), np.float32)
    lib.lrto_render_lambert(C.byref(s), C.byref(p), rays.ctypes.data, len(rays), L.ctypes.data, img.ctypes.data,
                            int(threads))
    del keep
    return img


def port_render_rgba8(arrays, rays, lights, background, preset=None, threads=os.cpu_count(), materials=None,
                      mat_ids=None, mat_offsets=None):
    """RGBA8 image of the eye rays `rays` (row-major pixels): nearest hit,
    the resolve of preset.render_mode with `lights` (LIGHT_DTYPE) and the
    renderer's COLORED materials (MATERIAL_DTYPE, ids, {start, size} per
    geometry) where the mode reads them, and tonemap."""
    from graphic_lab_task_b200._abi import LIGHT_DTYPE, MATERIAL_DTYPE
    lib = port_lib()
    if not hasattr(lib, "_rgba8_modes_bound"):
        lib.lrto_render_rgba8_modes.restype = None
        lib.lrto_render_rgba8_modes.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_uint64,
                                                C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_int]
        lib._rgba8_modes_bound = True
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    lt = np.ascontiguousarray(lights, dtype=LIGHT_DTYPE)
    bg = np.ascontiguousarray(background, dtype=np.float32)
    mats = None if materials is None else np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)
    ids = None if mat_ids is None else np.ascontiguousarray(mat_ids, dtype=np.uint32)
    offs = None if mat_offsets is None else np.ascontiguousarray(mat_offsets, dtype=np.uint32).reshape(-1)
    img = np.zeros(len(rays), np.uint32)
    ptr = lambda a: a.ctypes.data if a is not None and len(a) else None  # noqa: E731
    lib.lrto_render_rgba8_modes(C.byref(s), C.byref(p), rays.ctypes.data, len(rays), ptr(lt), len(lt),
                                bg.ctypes.data, ptr(mats), ptr(ids), ptr(offs), img.ctypes.data, int(threads))
    del keep
    return img


def port_render_rgba8_samples(arrays, sample_rays, resolve_rays, lights, background, preset, materials=None,
                              mat_ids=None, mat_offsets=None, transparency=False, max_layers=256,
                              threads=os.cpu_count()):
    """Render's sample loop: sample_rays is (samples, n, 8) (initEyeRay's
    point s of each pixel), resolve_rays (n, 8) the sample-0 rays the resolve
    uses; `transparency` takes the AnyHit path of DIFFUSE / LAMBERT / PHONG."""
    from graphic_lab_task_b200._abi import LIGHT_DTYPE, MATERIAL_DTYPE
    lib = port_lib()
    if not hasattr(lib, "_rgba8_ex_bound"):
        lib.lrto_render_rgba8_ex.restype = None
        lib.lrto_render_rgba8_ex.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_uint32,
                                             C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_int, C.c_uint32, C.c_void_p, C.c_int]
        lib._rgba8_ex_bound = True
    s, keep = arrays_to_struct(arrays)
    sr = np.ascontiguousarray(sample_rays, dtype=np.float32)
    rr = np.ascontiguousarray(resolve_rays, dtype=np.float32).reshape(-1, 8)
    n = len(rr)
    assert sr.size == sr.shape[0] * n * 8
    lt = np.ascontiguousarray(lights, dtype=LIGHT_DTYPE)
    bg = np.ascontiguousarray(background, dtype=np.float32)
    mats = None if materials is None else np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)
    ids = None if mat_ids is None else np.ascontiguousarray(mat_ids, dtype=np.uint32)
    offs = None if mat_offsets is None else np.ascontiguousarray(mat_offsets, dtype=np.uint32).reshape(-1)
    img = np.zeros(n, np.uint32)
    ptr = lambda a: a.ctypes.data if a is not None and len(a) else None  # noqa: E731
    lib.lrto_render_rgba8_ex(C.byref(s), C.byref(preset), sr.ctypes.data, sr.shape[0], rr.ctypes.data, n, ptr(lt),
                             len(lt), bg.ctypes.data, ptr(mats), ptr(ids), ptr(offs), int(bool(transparency)),
                             int(max_layers), img.ctypes.data, int(threads))
    del keep
    return img


def port_render_outline_border(arrays, sample_rays, resolve_rays, width, height, lights, background, preset,
                               threads=os.cpu_count()):
    """Render for OUTLINE_BORDER over a width x height image (row-major):
    sample_rays (samples, n, 8), resolve_rays (n, 8) the sample-0 rays."""
    from graphic_lab_task_b200._abi import LIGHT_DTYPE
    lib = port_lib()
    if not hasattr(lib, "_outline_bound"):
        lib.lrto_render_outline_border.restype = None
        lib.lrto_render_outline_border.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_uint32,
                                                   C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32,
                                                   C.c_void_p, C.c_void_p, C.c_int]
        lib._outline_bound = True
    s, keep = arrays_to_struct(arrays)
    sr = np.ascontiguousarray(sample_rays, dtype=np.float32)
    rr = np.ascontiguousarray(resolve_rays, dtype=np.float32).reshape(-1, 8)
    n = width * height
    assert len(rr) == n and sr.size == sr.shape[0] * n * 8
    lt = np.ascontiguousarray(lights, dtype=LIGHT_DTYPE)
    bg = np.ascontiguousarray(background, dtype=np.float32)
    img = np.zeros(n, np.uint32)
    lib.lrto_render_outline_border(C.byref(s), C.byref(preset), sr.ctypes.data, sr.shape[0], rr.ctypes.data, width,
                                   height, lt.ctypes.data if len(lt) else None, len(lt), bg.ctypes.data,
                                   img.ctypes.data, int(threads))
    del keep
    return img


def port_fill_gbuffer_transparency(arrays, rays, materials, mat_ids, mat_offsets, background, max_layers=256,
                                   preset=None, threads=os.cpu_count()):
    """AnyHit's transparency loop per eye ray (rays: row-major pixels).
    Returns (transparency float4 per ray, last hits, rays that hit the layer bound)."""
    from graphic_lab_task_b200._abi import MATERIAL_DTYPE
    lib = port_lib()
    if not hasattr(lib, "_transp_bound"):
        lib.lrto_fill_gbuffer_transparency.restype = C.c_uint64
        lib.lrto_fill_gbuffer_transparency.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p,
                                                       C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_uint32, C.c_void_p, C.c_void_p, C.c_int]
        lib._transp_bound = True
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    mats = np.ascontiguousarray(materials, dtype=MATERIAL_DTYPE)
    ids = np.ascontiguousarray(mat_ids, dtype=np.uint32)
    offs = np.ascontiguousarray(mat_offsets, dtype=np.uint32).reshape(-1)
    bg = np.ascontiguousarray(background, dtype=np.float32)
    transp = np.zeros((len(rays), 4), np.float32)
    hits = np.zeros(len(rays), HIT_DTYPE)
    capped = lib.lrto_fill_gbuffer_transparency(C.byref(s), C.byref(p), rays.ctypes.data, len(rays),
                                                mats.ctypes.data if len(mats) else None,
                                                ids.ctypes.data if len(ids) else None,
                                                offs.ctypes.data if len(offs) else None, bg.ctypes.data,
                                                int(max_layers), transp.ctypes.data, hits.ctypes.data, int(threads))
    del keep
    return transp, hits, int(capped)


def port_adjoint_fp64(arrays, rays, light, dimage, preset=None):
    """FP64 adjoint of the Lambert render w.r.t. the SBS float values."""
    port_render_lambert(arrays, np.zeros((0, 8), np.float32), light, preset)  # binds the signatures
    lib = port_lib()
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    L = np.ascontiguousarray(light, dtype=np.float32)
    di = np.ascontiguousarray(dimage, dtype=np.float32)
    grad = np.zeros(len(arrays["sdfSBSDataF"]), np.float64)
    lib.lrto_adjoint_lambert_fp64(C.byref(s), C.byref(p), rays.ctypes.data, len(rays), L.ctypes.data,
                                  di.ctypes.data, grad.ctypes.data)
    del keep
    return grad


def port_fd_model_fp64(arrays, rays, light, dimage, keys, h=1e-6, preset=None, threads=os.cpu_count(),
                       shape=False):
    """Central differences (FP64 surface model of each hit voxel) of
    sum_i dimage[i] * I_i w.r.t. the value indices `keys`.  With shape=True
    also returns, per key, the smallest |cos(grad f, d)| and n . L over the
    pixels whose hit voxel has that value as a corner."""
    lib = port_lib()
    if not hasattr(lib, "_fd_bound"):
        lib.lrto_fd_model_fp64_shape.restype = None
        lib.lrto_fd_model_fp64_shape.argtypes = [C.POINTER(SceneArrays), C.POINTER(Preset), C.c_void_p, C.c_uint64,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_double,
                                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        lib._fd_bound = True
    s, keep = arrays_to_struct(arrays)
    p = preset if preset is not None else parity_preset()
    rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 8)
    L = np.ascontiguousarray(light, dtype=np.float32)
    di = np.ascontiguousarray(dimage, dtype=np.float32)
    order = np.argsort(keys)
    k = np.ascontiguousarray(np.asarray(keys, np.uint32)[order])
    out = np.zeros(len(k), np.float64)
    mc = np.zeros(len(k), np.float64)
    mn = np.zeros(len(k), np.float64)
    lib.lrto_fd_model_fp64_shape(C.byref(s), C.byref(p), rays.ctypes.data, len(rays), L.ctypes.data,
                                 di.ctypes.data, k.ctypes.data, len(k), float(h), out.ctypes.data,
                                 mc.ctypes.data if shape else None, mn.ctypes.data if shape else None, int(threads))
    del keep
    res = np.empty_like(out)
    res[order] = out
    if not shape:
        return res
    rc, rn = np.empty_like(mc), np.empty_like(mn)
    rc[order] = mc
    rn[order] = mn
    return res, rc, rn


def ref_trace(arrays, rays, preset=None, threads=1, fast=False):
    """Trace already-flattened arrays with the reference BVHRT."""
    sc = RefScene(fast=fast, preset=preset)
    try:
        sc.import_arrays(arrays)
        return sc.trace(rays, threads=threads)
    finally:
        sc.close()

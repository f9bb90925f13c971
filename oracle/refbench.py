"""The reference arm of bench.py (BASELINE ONLY; the product never imports it).

`bench.py --impl reference` times the reference's own CPU implementation of
the benchmark's ray query on the host cores, end to end through the
reference's own code: its host build (BVHRT::AddGeom_SdfSBS, AddInstance,
CommitScene with the cbvh pipeline), its preset, its camera (LiteMath lookAt /
perspectiveMatrix, MultiRenderer::UpdateCamera) and eye rays
(MultiRenderer::initEyeRay), and BVHRT::RayQuery_NearestHit with OpenMP over
rays — all compiled from the reference's sources into
oracle/_ref/liblrt_ref_fast.so with its Release-style flags.  The seeded
sparse brick set comes from oracle/_build/liblrt_workloads.so, the benchmark
input generator compiled on its own.  Nothing here loads the product library
or imports the product package.
"""
import ctypes as C
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_FAST_SO = os.path.join(HERE, "_ref", "liblrt_ref_fast.so")
WL_SO = os.path.join(HERE, "_build", "liblrt_workloads.so")
SBS_HEADER_BYTES = 16  # SdfSBSHeader (sdf/simple/sdf_simple_shared.h)
SBS_NODE_BYTES = 16    # SdfSBSNode
HIT_BYTES = 32         # CRT_Hit


def available():
    """None when both libraries exist, else the reason."""
    for p in (REF_FAST_SO, WL_SO):
        if not os.path.exists(p):
            return "%s not built (make -C oracle ref wl)" % os.path.relpath(p, os.path.dirname(HERE))
    return None


def _libs():
    vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
    wl = C.CDLL(WL_SO)
    wl.lrt_wl_spheres.restype = C.c_int
    wl.lrt_wl_spheres.argtypes = [u32, C.c_float, C.c_float, C.c_float, u64, vp]
    wl.lrt_wl_sbs_from_spheres.restype = C.c_int
    wl.lrt_wl_sbs_from_spheres.argtypes = [vp, u32, u32, u32, u32, vp, vp, vp, vp, vp, vp, vp]
    ref = C.CDLL(REF_FAST_SO)
    ref.lrtr_create.restype = vp
    ref.lrtr_create.argtypes = [C.c_char_p, C.c_char_p]
    ref.lrtr_add_sbs.restype = u32
    ref.lrtr_add_sbs.argtypes = [vp, vp, vp, u64, vp, u64, vp, u64]
    ref.lrtr_add_instance.restype = u32
    ref.lrtr_add_instance.argtypes = [vp, u32, vp]
    ref.lrtr_renderer_create.restype = vp
    for fn, args in (("lrtr_destroy", [vp]), ("lrtr_set_parity_preset", [vp]), ("lrtr_commit", [vp]),
                     ("lrtr_trace", [vp, vp, vp, u64, C.c_int]), ("lrtr_renderer_create", [vp]),
                     ("lrtr_renderer_destroy", [vp]),
                     ("lrtr_renderer_look_at", [vp, vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float]),
                     ("lrtr_renderer_eye_rays", [vp, u32, u32, u32, vp])):
        getattr(ref, fn).argtypes = args
        if fn != "lrtr_renderer_create":
            getattr(ref, fn).restype = None
    return wl, ref


def _check(rc, what):
    if rc != 0:
        raise RuntimeError("%s failed with status %d" % (what, rc))


def sbs_model(wl, n_spheres, sphere_seed, grid, brick, pad):
    """The benchmark's sparse brick set: union of `n_spheres` seeded spheres
    (centres U[-0.8, 0.8]^3, radii U[0.05, 0.3]) on a virtual grid^3."""
    sph = np.zeros((n_spheres, 4), np.float32)
    _check(wl.lrt_wl_spheres(n_spheres, 0.8, 0.05, 0.3, sphere_seed, sph.ctypes.data), "lrt_wl_spheres")
    nn, nv, nf = C.c_uint64(), C.c_uint64(), C.c_uint64()
    _check(wl.lrt_wl_sbs_from_spheres(sph.ctypes.data, n_spheres, grid, brick, pad, None, None, None, None,
                                      C.byref(nn), C.byref(nv), C.byref(nf)), "lrt_wl_sbs_from_spheres")
    header = np.zeros(SBS_HEADER_BYTES, np.uint8)
    nodes = np.zeros(nn.value * SBS_NODE_BYTES, np.uint8)
    values = np.zeros(nv.value, np.uint32)
    values_f = np.zeros(nf.value, np.float32)
    _check(wl.lrt_wl_sbs_from_spheres(sph.ctypes.data, n_spheres, grid, brick, pad, header.ctypes.data,
                                      nodes.ctypes.data, values.ctypes.data, values_f.ctypes.data, C.byref(nn),
                                      C.byref(nv), C.byref(nf)), "lrt_wl_sbs_from_spheres")
    return header, nodes, int(nn.value), values, values_f


def run(width, height, grid, brick, pad, n_spheres, sphere_seed, tmin, tmax, steps, warmup, seconds=60.0,
        threads=None):
    """Builds the scene and the rays with the reference's code, then times
    `steps` traces of a strided sample of the image's rays sized so that the
    whole run takes about `seconds`.  Returns a dict of the measurement."""
    wl, ref = _libs()
    threads = threads or os.cpu_count()
    header, nodes, nn, values, values_f = sbs_model(wl, n_spheres, sphere_seed, grid, brick, pad)
    h = ref.lrtr_create(b"cbvh_embree2", b"SuperTreeletAlignedMerged4")
    if not h:
        raise RuntimeError("CreateSceneRT failed")
    r = None
    try:
        ref.lrtr_set_parity_preset(h)
        g = ref.lrtr_add_sbs(h, header.ctypes.data, nodes.ctypes.data, nn, values.ctypes.data, len(values),
                             values_f.ctypes.data, len(values_f))
        identity = np.eye(4, dtype=np.float32).reshape(16)
        ref.lrtr_add_instance(h, g, identity.ctypes.data)
        ref.lrtr_commit(h)
        # the camera at (0, 0, 3) looking at the origin, 60 degree fovy,
        # MultiRenderer's zNear 0.01 / zFar 100 (MultiRenderer_host.cpp:1078)
        r = ref.lrtr_renderer_create(h)
        eye = np.array([0, 0, 3], np.float32)
        center = np.zeros(3, np.float32)
        up = np.array([0, 1, 0], np.float32)
        ref.lrtr_renderer_look_at(r, eye.ctypes.data, center.ctypes.data, up.ctypes.data, 60.0, width / height,
                                  0.01, 100.0)
        rays = np.zeros((width * height, 8), np.float32)
        ref.lrtr_renderer_eye_rays(r, width, height, 0, rays.ctypes.data)
        rays[:, 3] = tmin  # the workload's interval (initEyeRay's own is 1e-9 .. 1e9)
        rays[:, 7] = tmax
        n = len(rays)

        def trace(x):
            x = np.ascontiguousarray(x)
            hits = np.zeros(len(x) * HIT_BYTES, np.uint8)
            ref.lrtr_trace(h, x.ctypes.data, hits.ctypes.data, len(x), threads)
            return hits

        probe = rays[:: max(1, n // 32768)]
        t0 = time.perf_counter()
        trace(probe)
        rate = len(probe) / max(time.perf_counter() - t0, 1e-6)
        per_step = max(len(probe), min(n, int(rate * seconds / max(1, steps + warmup))))
        sample = np.ascontiguousarray(rays[np.linspace(0, n - 1, per_step).astype(np.int64)])
        for _ in range(warmup):
            trace(sample[: max(1, per_step // 8)])
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            trace(sample)
            times.append(time.perf_counter() - t0)
        ms = 1e3 * sum(times) / len(times)
        return {"value": per_step / (ms * 1e-3) / 1e6, "ms_per_step": ms, "rays_per_step": per_step, "threads": threads,
                "sample": "%d of %d rays (strided over the image) per step; scene, preset, camera and eye rays built "
                          "by the reference's own code; OpenMP over rays" % (per_step, n)}
    finally:
        if r:
            ref.lrtr_renderer_destroy(r)
        ref.lrtr_destroy(h)

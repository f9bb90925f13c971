"""The reference-side drop-in, compiled and run: the BVHRT_B200 subclass of
INTEGRATION.md (oracle/ref/bvhrt_b200.cpp) built against the reference's
headers and objects and linked against liblrt_b200.so.  Scenes go through
the reference's own AddGeom_* / AddInstance / CommitScene; the overridden
CommitScene uploads the reference's arrays; RayQuery_NearestHit,
RayQuery_AnyHit and the batched query run on the GPU.  Every hit equals the
reference CPU path on the same scene bit for bit."""
import os

import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import workloads as wl
from helpers import MISS, RefBuilder, bit_equal, hit_summary

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not po.dropin_available(), reason="drop-in build absent (make -C oracle dropin)")]


class DropInBuilder(RefBuilder):
    def __init__(self):
        self.ref = po.DropInScene()


def _mixed(b, seed=0):
    sph = wl.spheres(24, seed=40 + seed)
    v, t = wl.noisy_sphere(48, seed=seed)
    gm = b.AddGeom_Triangles3f(v, t)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64)
    gb = b.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    go = b.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 5))
    gs = b.AddGeom_SdfSVS(wl.svs_from_spheres(sph, 5))
    for i, m in enumerate(wl.random_instances(48, seed=seed, scale=(0.2, 0.5), trans=1.4)):
        b.AddInstance([gm, gb, go, gs][i % 4], m)
    return b.CommitScene()


@pytest.mark.parametrize("seed", [0, 1])
def test_dropin_subclass_traces_like_the_reference(cuda, seed):
    gpu = _mixed(DropInBuilder(), seed)
    cpu = _mixed(RefBuilder(), seed)
    # the subclass keeps the reference's scene assembly: identical arrays
    a, b = gpu.export(), cpu.export()
    for k in a:
        assert a[k].tobytes() == b[k].tobytes(), k
    rays = wl.eye_rays_host(wl.camera((0.3, 0.8, 3.4), width=160, height=120))
    rays = np.concatenate([rays, rays[::7] * np.array([1, 1, 1, 1, 1, 1, 1, -1], np.float32)])  # stop-on-first
    want = cpu.trace(rays, threads=os.cpu_count())
    got = gpu.trace_batch(rays)                            # RayQuery_NearestHitBatch
    assert bit_equal(got, want).all(), hit_summary(got, want)
    assert (want["primId"] != MISS).sum() > 3000
    some = rays[::97]
    one = gpu.trace(some, threads=1)                       # the virtual RayQuery_NearestHit, one ray per call
    sub = np.ascontiguousarray(want[::97])
    assert bit_equal(one, sub).all(), hit_summary(one, sub)


def test_dropin_sbs_benchmark_model(cuda):
    """The benchmark's SBS (512^3 virtual grid) through the subclass, all
    1920x1080 rays in one batched query."""
    sph = wl.spheres(64, seed=1)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=512)
    gpu, cpu = DropInBuilder(), RefBuilder()
    for b in (gpu, cpu):
        b.AddInstance(b.AddGeom_SdfSBS(hdr, nodes, vals, vf), wl.IDENTITY)
    gpu, cpu = gpu.CommitScene(), cpu.CommitScene()
    rays = wl.eye_rays_host(wl.camera((0, 0, 3), width=1920, height=1080))
    got = gpu.trace_batch(rays)
    want = cpu.trace(rays, threads=os.cpu_count())
    assert bit_equal(got, want).all(), hit_summary(got, want)

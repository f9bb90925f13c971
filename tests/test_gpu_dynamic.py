"""Dynamic instances: UpdateInstance followed by CommitScene rebuilds the
TLAS and writes only the TLAS and the instances to the device; traces then
equal the oracle on the exported arrays and a scene built with the new
transforms from the start, and a batched-camera graph captured before the
update is re-captured."""
import time

import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import HIT_DTYPE, SceneRT, workloads as wl
from graphic_lab_task_b200.lrt import CameraBatch
from helpers import MISS, bit_equal, hit_summary

pytestmark = pytest.mark.gpu


def _build(mats, sph):
    sc = SceneRT()
    v, t = wl.noisy_sphere(40, seed=2)
    gm = sc.AddGeom_Triangles3f(v, t)
    go = sc.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 5))
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64)
    gb = sc.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    for i, m in enumerate(mats):
        sc.AddInstance([gm, go, gb][i % 3], m)
    return sc


def test_update_instances_then_commit(cuda):
    sph = wl.spheres(24, seed=4)
    mats = wl.random_instances(96, seed=7, scale=(0.1, 0.4), trans=1.5)
    new = wl.random_instances(96, seed=8, scale=(0.1, 0.4), trans=1.5)
    sc = _build(mats, sph)
    t0 = time.perf_counter()
    sc.CommitScene()
    full_s = time.perf_counter() - t0
    rays = wl.eye_rays_host(wl.camera((0.5, 0.7, 3.5), width=160, height=120))
    before = sc.RayQuery_NearestHitBatch(rays)
    final = list(mats)
    for i in range(0, 96, 3):
        sc.UpdateInstance(i, new[i], update_normal_matrix=True)
        final[i] = new[i]
    t0 = time.perf_counter()
    sc.CommitScene()
    update_s = time.perf_counter() - t0
    got = sc.RayQuery_NearestHitBatch(rays)
    want = po.port_trace(sc.export_arrays(), rays)
    assert bit_equal(got, want).all(), hit_summary(got, want)
    assert not bit_equal(got, before).all()
    fresh = _build(final, sph)
    fresh.CommitScene()
    again = fresh.RayQuery_NearestHitBatch(rays)
    assert bit_equal(got, again).all(), hit_summary(got, again)
    print("commit: full %.1f ms, instances only %.1f ms" % (1e3 * full_s, 1e3 * update_s))
    # clear the instances and add a different number of them: new TLAS and instance buffers
    sc.ClearScene()
    for i, m in enumerate(final[:50]):
        sc.AddInstance([0, 1, 2][i % 3], m)
    sc.CommitScene()
    got = sc.RayQuery_NearestHitBatch(rays)
    assert bit_equal(got, po.port_trace(sc.export_arrays(), rays)).all()


def test_batched_graph_follows_instance_updates(cuda):
    torch = cuda
    sph = wl.spheres(24, seed=4)
    mats = wl.random_instances(30, seed=7, scale=(0.1, 0.4), trans=1.2)
    sc = _build(mats, sph)
    sc.CommitScene()
    cams = wl.sphere_cameras(4, radius=3.0, res_min=64, res_max=96, seed=3)
    b = CameraBatch(sc, cams)
    hb = torch.zeros(b.total_rays * 8, dtype=torch.float32, device="cuda")
    b.trace(hb.data_ptr())
    b.sync()
    new = wl.random_instances(30, seed=9, scale=(0.1, 0.4), trans=1.2)
    for i in range(0, 30, 2):
        sc.UpdateInstance(i, new[i], update_normal_matrix=True)
    sc.CommitScene()
    b.trace(hb.data_ptr())
    b.sync()
    got = hb.cpu().numpy().view(HIT_DTYPE)
    want = np.concatenate([sc.RayQuery_NearestHitBatch(wl.eye_rays_host(c)) for c in cams])
    assert bit_equal(got, want).all(), hit_summary(got, want)
    assert (want["primId"] != MISS).sum() > 100
    b.close()

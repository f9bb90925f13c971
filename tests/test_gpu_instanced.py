"""Incoherent two-level workload: many instances of meshes and frame-octree
SDFs, primary rays and a second wavefront of cosine-weighted bounce rays, all
bit-identical to the oracle."""
import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import HIT_DTYPE, SceneRT, workloads as wl
from helpers import MISS, bit_equal, hit_summary

pytestmark = pytest.mark.gpu


def _bounce(torch, sc, rays_np, hits_t, seed=11):
    R = torch.from_numpy(rays_np).cuda()
    B = torch.empty_like(R)
    sc.generate_bounce_rays(R.data_ptr(), hits_t.data_ptr(), len(rays_np), seed, B.data_ptr())
    torch.cuda.synchronize()
    return B.cpu().numpy().reshape(-1, 8)


@pytest.mark.parametrize("scale", ["reduced", "full"])
def test_instanced_primary_and_bounce(cuda, scale):
    torch = cuda
    sc = SceneRT()
    if scale == "reduced":
        wl.build_instanced(sc, mesh_tris=(2000, 8000, 20000), octree_depth=6, n_instances=256)
        w = h = 256
    else:
        wl.build_instanced(sc)
        w = h = 4096
    sc.CommitScene()
    rays = wl.eye_rays_host(wl.camera(wl.INSTANCED_EYE, width=w, height=h))
    R = torch.from_numpy(rays).cuda()
    H = torch.empty(len(rays) * 8, dtype=torch.float32, device="cuda")
    sc.trace_device(R.data_ptr(), H.data_ptr(), len(rays))
    sc.sync()
    prim = H.cpu().numpy().view(HIT_DTYPE)
    hit = prim["primId"] != MISS
    assert hit.mean() > 0.05
    types = set((prim["geomId"][hit] >> 24).tolist())
    assert types == {0, 3}
    bounce = _bounce(torch, sc, rays, H)
    valid = ~np.isnan(bounce[:, 0])
    assert np.array_equal(valid, hit)
    d = bounce[valid, 4:7]
    assert np.allclose(np.linalg.norm(d, axis=1), 1, atol=1e-5)
    Bv = torch.from_numpy(np.ascontiguousarray(bounce[valid])).cuda()
    HB = torch.empty(len(Bv) * 8, dtype=torch.float32, device="cuda")
    sc.trace_device(Bv.data_ptr(), HB.data_ptr(), len(Bv))
    sc.sync()
    bh = HB.cpu().numpy().view(HIT_DTYPE)
    arrays = sc.export_arrays()
    if scale == "reduced":
        sel_p, sel_b = np.arange(len(rays)), np.arange(len(Bv))
    else:  # the oracle checks strided samples of the 16.8M primary and the bounce rays
        sel_p = np.unique(np.linspace(0, len(rays) - 1, 20000).astype(np.int64))
        sel_b = np.unique(np.linspace(0, len(Bv) - 1, 20000).astype(np.int64))
    want_p = po.port_trace(arrays, rays[sel_p])
    assert bit_equal(prim[sel_p], want_p).all(), hit_summary(prim[sel_p], want_p)
    bv = bounce[valid]
    want_b = po.port_trace(arrays, bv[sel_b])
    assert bit_equal(bh[sel_b], want_b).all(), hit_summary(bh[sel_b], want_b)
    # the NaN rays of the misses miss
    nan_rays = bounce[~valid][:256]
    if len(nan_rays):
        got = sc.RayQuery_NearestHitBatch(nan_rays)
        assert np.all(got["primId"] == MISS)

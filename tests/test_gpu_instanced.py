"""Incoherent two-level workload: many instances of meshes and frame-octree
SDFs, primary rays and a second wavefront of cosine-weighted bounce rays.
Every ray is bit-identical to the oracle on the product's arrays, and within
the specification's tolerance (bit-identical apart from near ties) of the
reference's own stock build of the same scene."""
import os

import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import HIT_DTYPE, SceneRT, workloads as wl
from helpers import MISS, RefBuilder, assert_within_spec, bit_equal, bounce_coherence_keys, hit_summary

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
    kw = dict(mesh_tris=(2000, 8000, 20000), octree_depth=6, n_instances=256) if scale == "reduced" else {}
    w = h = 256 if scale == "reduced" else 4096
    sc = SceneRT()
    wl.build_instanced(sc, **kw)
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
    bv = np.ascontiguousarray(bounce[valid])
    Bv = torch.from_numpy(bv).cuda()
    HB = torch.empty(len(Bv) * 8, dtype=torch.float32, device="cuda")
    sc.trace_device(Bv.data_ptr(), HB.data_ptr(), len(Bv))
    sc.sync()
    bh = HB.cpu().numpy().view(HIT_DTYPE)
    # every primary and every bounce ray against the oracle on the product's arrays
    arrays = sc.export_arrays()
    want_p = po.port_trace(arrays, rays)
    assert bit_equal(prim, want_p).all(), hit_summary(prim, want_p)
    want_b = po.port_trace(arrays, bv)
    assert bit_equal(bh, want_b).all(), hit_summary(bh, want_b)
    if po.ref_available():
        # the same scene assembled by the reference's own host code
        rb = RefBuilder()
        wl.build_instanced(rb, **kw)
        ref = rb.CommitScene()
        assert ref.export()["instanceData"]["transformInv"].tobytes() == arrays["instanceData"]["transformInv"].tobytes()
        rep_p = assert_within_spec(prim, ref.trace(rays, threads=os.cpu_count()), what="primary %dx%d" % (w, h),
                                   tree_ref=lambda idx: po.ref_trace(arrays, rays[idx]))
        rep_b = assert_within_spec(bh, ref.trace(bv, threads=os.cpu_count()), what="bounce",
                                   tree_ref=lambda idx: po.ref_trace(arrays, bv[idx]))
        print("reference build: primary %d/%d bit-identical (%d near ties, %d tree-order), bounce %d/%d "
              "(%d near ties, %d tree-order)" % (rep_p["bit_identical"], len(rays), rep_p["ties"],
                                                 rep_p["tree_order"], rep_b["bit_identical"], len(bv), rep_b["ties"],
                                                 rep_b["tree_order"]))
    # the NaN rays of the misses miss
    nan_rays = bounce[~valid][:256]
    if len(nan_rays):
        got = sc.RayQuery_NearestHitBatch(nan_rays)
        assert np.all(got["primId"] == MISS)


@pytest.mark.parametrize("n", [1, 2047, 2049, 300001])
def test_compacted_bounce_rays_equal_the_full_generator(cuda, n):
    """lrt_generate_bounce_rays_compact packs the bounce rays of the hits in
    ray order: they equal the full generator's rays at the hit positions,
    the index map is the list of hit rays and the device count their number."""
    torch = cuda
    sc = SceneRT()
    wl.build_instanced(sc, mesh_tris=(2000, 8000, 20000), octree_depth=6, n_instances=256)
    sc.CommitScene()
    rays = wl.eye_rays_host(wl.camera(wl.INSTANCED_EYE, width=600, height=501))[:n]
    R = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    H = torch.empty(n * 8, dtype=torch.float32, device="cuda")
    sc.trace_device(R.data_ptr(), H.data_ptr(), n)
    full = torch.empty(n * 8, dtype=torch.float32, device="cuda")
    sc.generate_bounce_rays(R.data_ptr(), H.data_ptr(), n, 5, full.data_ptr())
    comp = torch.full((n * 8,), -7.0, dtype=torch.float32, device="cuda")
    idx = torch.zeros(n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    sc.generate_bounce_rays_compact(R.data_ptr(), H.data_ptr(), n, 5, comp.data_ptr(), idx.data_ptr(), cnt.data_ptr())
    sc.sync()
    hits = H.cpu().numpy().view(HIT_DTYPE)
    want_idx = np.nonzero(hits["primId"] != MISS)[0]
    k = int(cnt.item())
    assert k == len(want_idx)
    assert np.array_equal(idx.cpu().numpy()[:k].astype(np.int64), want_idx)
    f = full.cpu().numpy().reshape(-1, 8)
    c = comp.cpu().numpy().reshape(-1, 8)
    assert np.array_equal(c[:k].view(np.uint32), f[want_idx].view(np.uint32))
    assert np.all(c[k:] == -7.0)  # nothing written past the count


@pytest.mark.parametrize("n", [0, 1, 2047, 300001])
def test_sorted_bounce_rays_are_the_compact_ones_in_key_order(cuda, n):
    """lrt_generate_bounce_rays_sorted returns the compacted bounce rays and
    their index map permuted by a stable sort of the coherence key (restated
    in numpy), the same count, and traces of the sorted rays equal the
    oracle's."""
    torch = cuda
    sc = SceneRT()
    wl.build_instanced(sc, mesh_tris=(2000, 8000, 20000), octree_depth=6, n_instances=256)
    sc.CommitScene()
    rays = wl.eye_rays_host(wl.camera(wl.INSTANCED_EYE, width=600, height=501))[:n]
    m = max(n, 1)
    R = torch.from_numpy(np.ascontiguousarray(rays)).cuda() if n else torch.zeros(8, device="cuda")
    H = torch.empty(m * 8, dtype=torch.float32, device="cuda")
    sc.trace_device(R.data_ptr(), H.data_ptr(), n)
    comp = torch.full((m * 8,), -7.0, dtype=torch.float32, device="cuda")
    idx = torch.zeros(m, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    sc.generate_bounce_rays_compact(R.data_ptr(), H.data_ptr(), n, 5, comp.data_ptr(), idx.data_ptr(), cnt.data_ptr())
    srt = torch.full((m * 8,), -7.0, dtype=torch.float32, device="cuda")
    sidx = torch.zeros(m, dtype=torch.int32, device="cuda")
    scnt = torch.full((1,), 99, dtype=torch.int64, device="cuda")
    for _ in range(2):  # the second call reuses the scene's sort scratch
        sc.generate_bounce_rays_sorted(R.data_ptr(), H.data_ptr(), n, 5, srt.data_ptr(), sidx.data_ptr(),
                                       scnt.data_ptr())
    sc.sync()
    k = int(cnt.item())
    assert int(scnt.item()) == k
    c = comp.cpu().numpy().reshape(-1, 8)[:k]
    ci = idx.cpu().numpy()[:k]
    order = np.argsort(bounce_coherence_keys(c, sc.export_arrays()["instanceData"]), kind="stable")
    got = srt.cpu().numpy().reshape(-1, 8)
    assert np.array_equal(got[:k].view(np.uint32), c[order].view(np.uint32))
    assert np.array_equal(sidx.cpu().numpy()[:k], ci[order])
    assert np.all(got[k:] == -7.0)  # nothing written past the count
    if k:
        if n > 2047:
            # consecutive sorted rays share their direction cell far more often than in ray order
            cells = bounce_coherence_keys(got[:k], sc.export_arrays()["instanceData"]) >> 18
            assert (cells[1:] == cells[:-1]).mean() > 0.9
        sel = np.unique(np.linspace(0, k - 1, min(k, 4000)).astype(np.int64))
        B = torch.from_numpy(np.ascontiguousarray(got[sel])).cuda()
        HB = torch.empty(len(sel) * 8, dtype=torch.float32, device="cuda")
        sc.trace_device(B.data_ptr(), HB.data_ptr(), len(sel))
        sc.sync()
        bh = HB.cpu().numpy().view(HIT_DTYPE)
        want = po.port_trace(sc.export_arrays(), got[sel])
        assert bit_equal(bh, want).all(), hit_summary(bh, want)

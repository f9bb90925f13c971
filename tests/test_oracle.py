"""The C restatement (oracle/lrt_oracle.c) against the reference's own golden
vectors, and — where the reference build exists — against the reference on
fresh scenes."""
import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import workloads as wl
from graphic_lab_task_b200._abi import COUNTER_NAMES
from helpers import MISS, bit_equal, golden_names, hit_summary, load_golden

GOLDEN = golden_names()


def test_golden_set_is_complete():
    for name in ("hand_triangle", "hand_brick", "mesh_small", "sbs_small", "instanced_mix", "ref_frame_octree",
                 "ref_svs_crop", "ref_sbs_crop", "solver_analytic", "solver_newton", "solver_it"):
        assert name in GOLDEN


@pytest.mark.parametrize("name", GOLDEN)
def test_port_matches_reference_golden(name):
    arrays, rays, want, preset = load_golden(name)
    got, cnt, limits = po.port_trace(arrays, rays, preset=preset, threads=4, counters=True)
    assert limits == 0
    assert bit_equal(got, want).all(), hit_summary(got, want)
    assert int(cnt[list(COUNTER_NAMES).index("hits")]) == int((want["primId"] != MISS).sum())


def test_hand_triangle_semantics():
    arrays, rays, want, _ = load_golden("hand_triangle")
    t = want["t"]
    assert t[0] == pytest.approx(1.0) and want["primId"][0] == 0
    assert want["primId"][2] == MISS           # t = 0.005 is inside the 0.01 leaf bias
    assert t[3] == pytest.approx(0.02)
    assert want["primId"][4] == MISS           # tfar = 0.5 before the triangle
    assert want["primId"][5] == 0              # any-hit ray still reports the hit
    assert want["primId"][9] == MISS


def test_planted_mistake_is_detected():
    """Moving one vertex of the golden mesh changes the oracle's answer."""
    arrays, rays, want, preset = load_golden("mesh_small")
    bad = {k: v.copy() for k, v in arrays.items()}
    first_hit = int(np.nonzero(want["primId"] != MISS)[0][0])
    g_off = int(bad["geomData"]["offset"][0][1])
    tri = int(want["primId"][first_hit])
    # the reordered triangle slot of that primitive
    slot = int(np.nonzero(bad["primIndices"] == tri)[0][0])
    vid = int(bad["indices"][3 * slot])
    bad["vertPos"][g_off + vid, :3] += np.float32(0.05)
    got = po.port_trace(bad, rays, preset=preset)
    assert not bit_equal(got, want).all()


@pytest.mark.skipif(not po.ref_available(), reason="reference build absent (make -C oracle ref)")
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_port_matches_reference_on_fresh_scenes(seed):
    rng = np.random.default_rng(seed)
    sph = wl.spheres(12, seed=100 + seed)
    v, t = wl.noisy_sphere(int(rng.integers(8, 30)), seed=seed)
    ref = po.RefScene()
    gm = ref.add_triangles(v, t)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    gb = ref.add_sbs(hdr, nodes, vals, vf)
    gs = ref.add_svs(wl.svs_from_spheres(sph, 4))
    for i, m in enumerate(wl.random_instances(7, seed=seed, scale=(0.3, 0.8), trans=1.2)):
        ref.add_instance([gm, gb, gs][i % 3], m)
    ref.commit()
    rays = wl.eye_rays_host(wl.camera((0.5, 1.0, 3.5), width=40, height=30))
    rays = np.concatenate([rays, rays[::3] * np.array([1, 1, 1, 1, 1, 1, 1, -1], np.float32)])
    want = ref.trace(rays)
    got = po.port_trace(ref.export(), rays)
    assert bit_equal(got, want).all(), hit_summary(got, want)


@pytest.mark.skipif(not po.ref_available(), reason="reference build absent (make -C oracle ref)")
@pytest.mark.parametrize("solver", [0, 1, 2, 3, 4])
def test_port_matches_reference_for_every_node_solver(solver):
    """ST, ANALYTIC (the reference's default), NEWTON, BBOX and IT inside
    SBS, frame-octree and SVS leaves, on a fresh scene."""
    from graphic_lab_task_b200._abi import parity_preset
    p = parity_preset()
    p.sdf_node_intersect = solver
    sph = wl.spheres(20, seed=40 + solver)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=48, brick_size=4, brick_pad=1)
    ref = po.RefScene(preset=p)
    gb = ref.add_sbs(hdr, nodes, vals, vf)
    go = ref.add_frame_octree(wl.frame_octree_from_spheres(sph, 5))
    gs = ref.add_svs(wl.svs_from_spheres(sph, 5))
    for i, m in enumerate(wl.random_instances(9, seed=50 + solver, scale=(0.4, 0.9), trans=1.2)):
        ref.add_instance([gb, go, gs][i % 3], m)
    ref.commit()
    rays = wl.eye_rays_host(wl.camera((0.2, 0.4, 4.0), width=96, height=96))
    want = ref.trace(rays, threads=4)
    got = po.port_trace(ref.export(), rays, preset=p)
    assert (want["primId"] != MISS).sum() > 500
    assert bit_equal(got, want).all(), hit_summary(got, want)


def transparency_tables(n_geoms_needing, prim_range=64, seed=0):
    """Materials for the transparency loop: four colours of different alpha,
    a textured one (composited as opaque black) and an opaque one; geometry g
    gets its own range of random material ids."""
    from graphic_lab_task_b200 import MATERIAL_COLORED, MATERIAL_DTYPE, MATERIAL_TEXTURED
    mats = np.zeros(6, MATERIAL_DTYPE)
    for k, (rgb, a) in enumerate([((1, 0, 0), 0.5), ((0, 1, 0), 0.3), ((0, 0, 1), 0.8), ((1, 1, 1), 0.05)]):
        mats[k] = (MATERIAL_COLORED, 0, 0.0, 0.5, (*rgb, a))
    mats[4] = (MATERIAL_TEXTURED, 3, 0.0, 0.5, (1, 1, 1, 1))
    mats[5] = (MATERIAL_COLORED, 0, 0.0, 0.5, (1, 1, 0, 1.0))
    rng = np.random.default_rng(seed)
    ids, offs = [], []
    for g in range(n_geoms_needing):
        size = int(rng.integers(1, prim_range))
        offs.append((len(ids), size))
        ids.extend(rng.choice([0, 1, 2, 3, 3, 3, 4, 5], size).tolist())
    return mats, np.array(ids, np.uint32), np.array(offs, np.uint32)


def test_transparency_loop_matches_its_statement():
    """The oracle's AnyHit loop (MultiRenderer.cpp:223-246) against the same
    loop written here over the oracle's nearest hit, ray by ray, in float32."""
    from test_builder import build_mixed
    sc, _ = build_mixed(seed=1)
    a = sc.export_arrays()
    mats, ids, offs = transparency_tables(len(a["geomData"]))
    bg = np.array([0.1, 0.2, 0.3, 1.0], np.float32)
    rays = wl.eye_rays_host(wl.camera((0.3, 0.9, 3.2), width=24, height=18))
    got_t, got_h, capped = po.port_fill_gbuffer_transparency(a, rays, mats, ids, offs, bg, threads=1)
    assert capped == 0
    f32 = np.float32
    for i, r in enumerate(rays):
        pn = r[:4].copy()
        tc = np.zeros(3, f32)
        alpha = f32(1)
        color = np.zeros(4, f32)
        while True:
            wa = f32(alpha * color[3])
            tc = (tc + wa * color[:3]).astype(f32)
            alpha = f32(alpha * f32(f32(1) - color[3]))
            h = po.port_trace(a, np.concatenate([pn, r[4:]])[None, :], threads=1)[0]
            typ, gid = int(h["geomId"]) >> 24, int(h["geomId"]) & 0xFFFFFF
            if h["primId"] == MISS:
                color = bg.copy()
            elif typ not in (11, 17):
                m = mats[ids[offs[gid][0] + int(h["primId"]) % offs[gid][1]]]
                color = m["base_color"].astype(f32) if m["type"] == 0 else np.array([0, 0, 0, 1], f32)
            pn[:3] = (pn[:3] + r[4:7] * f32(h["t"])).astype(f32)
            if not alpha > f32(0.01):
                break
        want = np.array([*tc, alpha], f32)
        assert got_t[i].view(np.uint32).tolist() == want.view(np.uint32).tolist(), (i, got_t[i], want)
        assert bit_equal(got_h[i:i + 1], h.reshape(1)).all()
    # several layers on some rays: the loop composited more than one surface
    assert (got_t[:, 3] < 0.99).sum() > 20 and np.unique(got_t[:, :3].round(4), axis=0).shape[0] > 10

"""Randomised parity sweep: seeded random two-level scenes of all leaf kinds,
random presets (render modes with and without normals or with the
sphere-tracing iteration count, SURFACE and VOLUME representation, the ST,
NEWTON, BBOX and IT node solvers) and random ray sets (camera rays, rays from
inside the scene, axis-parallel rays, any-hit rays, narrow [tmin, tfar]
windows).  Every hit of the exact build equals the oracle's bit for bit."""
import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import SceneRT, parity_preset, workloads as wl
from helpers import MISS, bit_equal, hit_summary

pytestmark = pytest.mark.gpu

RENDER_MODES = (1, 0, 10)  # LAMBERT_NO_TEX (normals), a mode without normals, ST_ITERATIONS
SOLVERS = (0, 2, 3, 4)     # ST, NEWTON, BBOX, IT (ANALYTIC is tolerance-tested elsewhere)


def _scene(rng, seed):
    sph = wl.spheres(int(rng.integers(4, 24)), seed=seed)
    kinds = [k for k in ("mesh", "octree", "svs", "sbs") if rng.random() < 0.7] or ["sbs"]
    p = parity_preset()
    p.render_mode = int(rng.choice(RENDER_MODES))
    p.sdf_node_intersect = int(rng.choice(SOLVERS))
    p.representation_mode = int(rng.integers(0, 2))
    sc = SceneRT(preset=p)
    geoms = []
    for k in kinds:
        if k == "mesh":
            v, t = wl.noisy_sphere(int(rng.integers(6, 40)), seed=seed)
            geoms.append(sc.AddGeom_Triangles3f(v, t))
        elif k == "octree":
            geoms.append(sc.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, int(rng.integers(3, 6)))))
        elif k == "svs":
            geoms.append(sc.AddGeom_SdfSVS(wl.svs_from_spheres(sph, int(rng.integers(3, 6)))))
        else:
            hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=int(rng.choice([16, 32, 48])),
                                                       brick_size=int(rng.choice([2, 4])), brick_pad=1)
            geoms.append(sc.AddGeom_SdfSBS(hdr, nodes, vals, vf))
    n_inst = int(rng.integers(1, 20))
    mats = wl.random_instances(n_inst, seed=seed, scale=(0.2, 0.9), trans=1.5)
    mats[0] = wl.IDENTITY.copy()  # object-space rays keep exact zeros
    if n_inst > 1:  # an axis-aligned, anisotropically scaled instance
        m = np.eye(4, dtype=np.float32)
        m[0, 0], m[1, 1], m[2, 2] = 0.5, 0.25, 0.75
        m[:3, 3] = rng.uniform(-1, 1, size=3)
        mats[1] = m.T.reshape(16).astype(np.float32)
    for i, m in enumerate(mats):
        sc.AddInstance(geoms[i % len(geoms)], m)
    sc.CommitScene()
    return sc, p


def _rays(rng):
    parts = [wl.eye_rays_host(wl.camera(tuple(rng.uniform(-0.5, 0.5, 2)) + (3.5,), width=48, height=40))]
    n = 1024
    o = rng.uniform(-1.5, 1.5, size=(n, 3))                    # origins inside and around the scene
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3], r[:, 4:7] = o, d
    r[:, 3], r[:, 7] = 1e-4, 1e9
    ax = rng.random(n) < 0.25                                   # axis-parallel directions
    k = rng.integers(0, 3, size=n)
    r[ax, 4:7] = 0.0
    r[ax, 4 + k[ax]] = rng.choice([-1.0, 1.0], size=ax.sum())
    win = rng.random(n) < 0.2                                    # narrow [tmin, tfar] windows
    r[win, 3] = rng.uniform(0.0, 1.0, size=win.sum())
    r[win, 7] = r[win, 3] + rng.uniform(0.0, 1.5, size=win.sum())
    anyh = rng.random(n) < 0.2                                   # any-hit queries
    r[anyh, 7] *= -1.0
    parts.append(r)
    return np.concatenate(parts).astype(np.float32)


@pytest.mark.parametrize("seed", range(40))
def test_random_scene_preset_and_rays(cuda, seed):
    rng = np.random.default_rng(1000 + seed)
    sc, p = _scene(rng, 1000 + seed)
    rays = _rays(rng)
    got = sc.RayQuery_NearestHitBatch(rays)
    want = po.port_trace(sc.export_arrays(), rays, preset=p)
    assert bit_equal(got, want).all(), (p.render_mode, p.sdf_node_intersect, p.representation_mode,
                                         hit_summary(got, want))
    assert (want["primId"] != MISS).any()

"""Seeded workload generators: sizes, determinism and agreement with the
analytic SDF (no GPU needed)."""
import numpy as np
import pytest

from graphic_lab_task_b200 import lib
from graphic_lab_task_b200 import workloads as wl


def test_noisy_sphere_sizes_and_noise():
    v, t = wl.noisy_sphere(317, seed=0)
    assert len(t) == 2 * 317 * 316 == 200344
    r = np.linalg.norm(v, axis=1)
    assert r.min() >= 0.95 - 1e-6 and r.max() <= 1.05 + 1e-6
    assert r.std() > 0.005                         # the noise is there
    v2, t2 = wl.noisy_sphere(317, seed=0)
    assert np.array_equal(v, v2) and np.array_equal(t, t2)
    assert t.max() == len(v) - 1
    assert wl.segments_for_triangles(200000) == 317


def test_spheres_ranges():
    s = wl.spheres(64, seed=1)
    assert np.all(np.abs(s[:, :3]) <= 0.8) and np.all((s[:, 3] >= 0.05) & (s[:, 3] <= 0.3))
    assert not np.array_equal(s, wl.spheres(64, seed=2))


def test_sbs_values_are_the_sdf():
    sph = wl.spheres(16, seed=3)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64, brick_size=8, brick_pad=1)
    assert hdr["aux_data"][0] == 4 << 24 and hdr["brick_size"][0] == 8 and hdr["brick_pad"][0] == 1
    v = 11
    L = lib()
    rng = np.random.default_rng(0)
    vox = 2.0 / 64
    for k in rng.choice(len(nodes), 8, replace=False):
        nd = nodes[k]
        bx, by, bz, G = nd["pos_xy"] >> 16, nd["pos_xy"] & 0xFFFF, nd["pos_z_lod_size"] >> 16, nd["pos_z_lod_size"] & 0xFFFF
        assert G == 8
        off = int(nd["data_offset"])
        for (a, b, c) in [(0, 0, 0), (1, 1, 1), (10, 3, 7), (5, 5, 5)]:
            idx = vals[off + (a * v + b) * v + c]
            p = -1 + vox * (np.array([bx, by, bz]) * 8 + np.array([a, b, c]) - 1)
            want = L.lrt_wl_sphere_sdf(sph.ctypes.data, len(sph), *map(float, p))
            assert vf[idx] == pytest.approx(want, abs=1e-6)
        # colour indices point at palette triples
        assert np.all(vals[off + v ** 3: off + v ** 3 + 8] % 3 == 0)
        assert np.all(vals[off + v ** 3: off + v ** 3 + 8] < 3 * len(sph))


def test_frame_octree_and_svs():
    sph = wl.spheres(8, seed=4)
    nodes = wl.frame_octree_from_spheres(sph, 5)
    assert nodes["offset"][0] == 1
    leaves = nodes[nodes["offset"] == 0]
    mixed = np.any(leaves["values"] <= 0, axis=1) & np.any(leaves["values"] > 0, axis=1)
    assert mixed.sum() > 100
    svs = wl.svs_from_spheres(sph, 5)
    assert len(svs) > 50 and np.all((svs["pos_z_lod_size"] & 0xFFFF) == 32)


def test_eye_rays_host():
    cam = wl.camera((0, 0, 3), width=64, height=48)
    r = wl.eye_rays_host(cam)
    assert r.shape == (64 * 48, 8)
    assert np.allclose(r[:, :3], [0, 0, 3], atol=1e-5)
    assert np.allclose(np.linalg.norm(r[:, 4:7], axis=1), 1, atol=1e-6)
    centre = r[24 * 64 + 32, 4:7]
    assert centre[2] < -0.99                        # looks at the origin
    # 60 degree vertical field of view
    top, bottom = r[32, 4:7], r[47 * 64 + 32, 4:7]
    ang = np.degrees(np.arccos(np.clip(np.dot(top, bottom), -1, 1)))
    assert ang == pytest.approx(60.0 * 47 / 48, abs=1.0)
    assert np.all(r[:, 3] == np.float32(1e-4)) and np.all(r[:, 7] == np.float32(1e9))


def test_instances_are_similarity_transforms():
    ms = wl.random_instances(16, seed=2)
    for m in ms:
        M = m.reshape(4, 4).T
        s = np.linalg.norm(M[:3, :3], axis=0)
        assert np.allclose(s, s[0], rtol=1e-5) and 0.05 <= s[0] <= 0.2
        assert np.all(np.abs(M[:3, 3]) <= 5)

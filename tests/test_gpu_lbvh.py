"""The device tree builder (BUILD_LOW, csrc/lbvh.cu): its trees have the
reference's array layouts, the kernels trace them bit-identically to the
oracle traversing the same arrays, and nearest triangle hits do not depend
on which builder made the tree."""
import sys
import time

import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import BUILD_HIGH, BUILD_LOW, SceneRT, workloads as wl
from helpers import MISS, bit_equal, check_blas_layout, check_tlas_layout, hit_summary

pytestmark = pytest.mark.gpu


def _mesh_scene(v, t, flags, build_name=None):
    sc = SceneRT(build_name=build_name) if build_name else SceneRT()
    sc.AddInstance(sc.AddGeom_Triangles3f(v, t, flags=flags), wl.IDENTITY)
    sc.CommitScene()
    return sc


@pytest.mark.parametrize("build_name", [None, "cbvh_embree4"])
def test_device_blas_layout_and_oracle_parity(cuda, build_name):
    v, t = wl.noisy_sphere(120, seed=5)
    sc = _mesh_scene(v, t, BUILD_LOW, build_name)
    a = sc.export_arrays()
    check_blas_layout(a, 0)
    pc = a["primIdCount"][a["startEnd"][0][0]:a["startEnd"][0][1]]
    counts = (pc >> 28) & 7
    cap = 4 if build_name else 2
    assert counts.min() >= 1 and counts.max() <= cap and counts.sum() == len(t)
    assert np.array_equal(a["indices"].reshape(-1, 3), t[a["primIndices"]])
    rays = wl.eye_rays_host(wl.camera((0.2, 0.4, 3), width=160, height=120))
    got = sc.RayQuery_NearestHitBatch(rays)
    want = po.port_trace(a, rays)
    assert bit_equal(got, want).all(), hit_summary(got, want)
    assert (got["primId"] != MISS).mean() > 0.2


def _coincident_mesh():
    """A small sphere plus 600 copies of one triangle and 300 of another:
    long runs of equal Morton codes, told apart by their sorted positions."""
    v, t = wl.noisy_sphere(24, seed=3)
    n = len(v)
    extra_v = np.array([[0.1, 0.1, 0.1], [0.2, 0.1, 0.1], [0.1, 0.2, 0.1], [-0.5, 0.3, 0.0], [-0.4, 0.3, 0.0],
                        [-0.5, 0.4, 0.0]], np.float32)
    extra_t = np.array([[n, n + 1, n + 2]] * 600 + [[n + 3, n + 4, n + 5]] * 300, np.uint32)
    return np.concatenate([v, extra_v]), np.concatenate([t, extra_t])


@pytest.mark.parametrize("build_name,cap", [(None, 2), ("cbvh_embree1", 1), ("cbvh_embree4", 4), ("cbvh_embree7", 7)])
@pytest.mark.parametrize("mesh", ["sphere", "coincident"])
def test_device_emission_equals_the_host_emitter(cuda, build_name, cap, mesh):
    """The triangle BLAS the device emits (pairs with their boxes, child and
    escape words; the leaf table; the triangle order) equals, bit for bit,
    the host emitter's layout of the same tree, modelled on the CPU from the
    same float32 Morton codes (tests/lbvh_model.py)."""
    import lbvh_model
    v, t = wl.noisy_sphere(40, seed=11) if mesh == "sphere" else _coincident_mesh()
    sc = _mesh_scene(v, t, BUILD_LOW, build_name)
    a = sc.export_arrays()
    pairs, table, order = lbvh_model.blas(v, t, cap)
    base = int(a["geomData"]["bvhOffset"][0])
    got = np.frombuffer(a["allNodePairs"].tobytes(), np.uint32).reshape(-1, 16)
    assert len(got) - base == len(pairs)
    assert np.array_equal(got[base:], pairs.view(np.uint32).reshape(-1, 16))
    a0, a1 = int(a["startEnd"][0][0]), int(a["startEnd"][0][1])
    assert np.array_equal(np.asarray(a["primIdCount"][a0:a1], np.uint32), table)
    assert np.array_equal(np.asarray(a["primIndices"][:len(order)], np.uint32), order)
    check_blas_layout(a, 0)


def test_device_and_sah_trees_give_the_same_triangle_hits(cuda):
    """Nearest triangle hits are a property of the mesh, not of the tree:
    every ray gets the same t from both builders; ids and coordinates differ
    only where two triangles tie at exactly that t (shared edges)."""
    v, t = wl.noisy_sphere(200, seed=6)
    rays = wl.eye_rays_host(wl.camera((0, 0, 3), width=256, height=256))
    low = _mesh_scene(v, t, BUILD_LOW).RayQuery_NearestHitBatch(rays)
    high = _mesh_scene(v, t, BUILD_HIGH).RayQuery_NearestHitBatch(rays)
    assert np.array_equal(low["t"].view(np.uint32), high["t"].view(np.uint32))
    same = bit_equal(low, high)
    assert same.mean() > 0.999, hit_summary(low, high)


def test_device_tlas_layout_and_oracle_parity(cuda):
    sph = wl.spheres(12, seed=210)
    sc = SceneRT()
    v, t = wl.noisy_sphere(24, seed=1)
    gm = sc.AddGeom_Triangles3f(v, t, flags=BUILD_LOW)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    gb = sc.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    go = sc.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 4))
    n_inst = 300
    for i, m in enumerate(wl.random_instances(n_inst, seed=9, scale=(0.05, 0.2), trans=1.5)):
        sc.AddInstance([gm, gb, go][i % 3], m)
    sc.CommitScene(options=BUILD_LOW)
    a = sc.export_arrays()
    check_tlas_layout(a["nodesTLAS"], n_inst)
    rays = wl.eye_rays_host(wl.camera((0.3, 0.5, 4.0), width=192, height=144))
    got = sc.RayQuery_NearestHitBatch(rays)
    want = po.port_trace(a, rays)
    assert bit_equal(got, want).all(), hit_summary(got, want)
    assert (got["primId"] != MISS).mean() > 0.1
    # a rebuilt TLAS after moving instances is still exact
    for k in range(0, n_inst, 7):
        m = wl.random_instances(1, seed=100 + k, scale=(0.05, 0.2), trans=1.5)[0]
        sc.UpdateInstance(k, m)
    sc.CommitScene(options=BUILD_LOW)
    a = sc.export_arrays()
    check_tlas_layout(a["nodesTLAS"], n_inst)
    got = sc.RayQuery_NearestHitBatch(rays)
    want = po.port_trace(a, rays)
    assert bit_equal(got, want).all(), hit_summary(got, want)


def test_device_aabb_blas(cuda):
    """Custom boxes (AddGeom_AABB): one box per leaf, every inner pair box
    containing the boxes below it."""
    rng = np.random.default_rng(3)
    n = 20000
    lo = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
    ext = rng.uniform(0.001, 0.05, (n, 3)).astype(np.float32)
    boxes = np.zeros((n, 8), np.float32)
    boxes[:, 0:3], boxes[:, 3] = lo, 1
    boxes[:, 4:7], boxes[:, 7] = lo + ext, 1
    sc = SceneRT()
    g = sc.AddGeom_AABB(7, boxes, flags=BUILD_LOW)
    a = sc.export_arrays()
    base = 0  # the only BLAS; AddGeom_AABB adds no geomData entry
    ids = check_blas_layout(a, g, base=base)
    assert len(ids) == n
    pairs = a["allNodePairs"]

    def box_of_subtree(k):
        """Min/max of the leaf boxes under pair k; checks containment on the way."""
        out_lo, out_hi = np.full(3, np.inf), np.full(3, -np.inf)
        for side in ("left", "right"):
            e = pairs[base + k][side]
            lo_ = int(e["leftOffset"])
            if lo_ & 0x80000000:
                if lo_ in (0xFFFFFFFF, 0x80000000):
                    continue
                b = boxes[a["primIdCount"][a["startEnd"][g][0] + (lo_ & 0x0FFFFFFF)]]
                sub_lo, sub_hi = b[0:3], b[4:7]
            else:
                sub_lo, sub_hi = box_of_subtree(lo_)
            assert np.all(e["boxMin"][:3] <= sub_lo) and np.all(e["boxMax"][:3] >= sub_hi)
            out_lo, out_hi = np.minimum(out_lo, sub_lo), np.maximum(out_hi, sub_hi)
        return out_lo, out_hi

    sys.setrecursionlimit(10000)
    box_of_subtree(0)


def test_device_build_is_much_faster_on_large_meshes(cuda):
    """Best of three builds each (the first device build of a process also
    loads the builder's kernels)."""
    v, t = wl.noisy_sphere(wl.segments_for_triangles(500000), seed=500000)
    times = {}
    for flags in (BUILD_LOW, BUILD_HIGH):
        best = float("inf")
        for _ in range(3):
            sc = SceneRT()
            t0 = time.perf_counter()
            sc.AddGeom_Triangles3f(v, t, flags=flags)
            best = min(best, time.perf_counter() - t0)
        times[flags] = best
    assert times[BUILD_LOW] < 0.5 * times[BUILD_HIGH], times

"""The product's scene assembly (csrc/scene.cpp): flattened arrays with the
reference's layouts, traced identically by the reference and the oracle, and
upload validation of malformed arrays (no GPU needed)."""
import os

import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import LrtError, SceneRT, workloads as wl
from helpers import (LEAF, MISS, RefBuilder, assert_within_spec, bit_equal, check_blas_layout, check_tlas_layout,
                     hit_summary)


def build_mixed(seed=0, n_inst=8, sc=None):
    """A mesh, an SBS, a frame octree and an SVS under `n_inst` random
    instances, assembled through `sc` (a SceneRT by default; a RefBuilder
    gives the same scene through the reference's own host code)."""
    sph = wl.spheres(12, seed=200 + seed)
    sc = SceneRT() if sc is None else sc
    v, t = wl.noisy_sphere(20, seed=seed)
    gm = sc.AddGeom_Triangles3f(v, t)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    gb = sc.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    go = sc.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 4))
    gs = sc.AddGeom_SdfSVS(wl.svs_from_spheres(sph, 4))
    for i, m in enumerate(wl.random_instances(n_inst, seed=seed, scale=(0.3, 0.8), trans=1.2)):
        sc.AddInstance([gm, gb, go, gs][i % 4], m)
    if isinstance(sc, RefBuilder):
        return sc.CommitScene(), (v, t)
    sc.CommitScene(host_only=True)
    return sc, (v, t)


def test_blas_layout_matches_reference_conventions():
    sc, (v, t) = build_mixed()
    a = sc.export_arrays()
    se = a["startEnd"]
    for g in range(len(a["geomData"])):
        check_blas_layout(a, g)
    # triangle leaves: primIdCount packs (start, count <= primsInLeaf), m_indices is the reordered index buffer
    g = 0
    pc = a["primIdCount"][se[g][0]:se[g][1]]
    counts = (pc >> 28) & 7
    assert counts.min() >= 1 and counts.max() <= 2 and counts.sum() == len(t)
    assert np.array_equal(a["indices"].reshape(-1, 3)[:len(t)], t[a["primIndices"][:len(t)]])


def test_tlas_escape_layout():
    sc, _ = build_mixed(n_inst=13)
    check_tlas_layout(sc.export_arrays()["nodesTLAS"], 13)


def test_single_instance_tlas_is_one_leaf():
    sc = SceneRT()
    v, t = wl.noisy_sphere(8)
    sc.AddInstance(sc.AddGeom_Triangles3f(v, t), wl.IDENTITY)
    sc.CommitScene(host_only=True)
    n = sc.export_arrays()["nodesTLAS"]
    assert len(n) == 1 and n[0]["leftOffset"] == LEAF and n[0]["escapeIndex"] == 0xFFFFFFFF


@pytest.mark.parametrize("seed", [0, 1])
def test_product_arrays_trace_like_reference(seed):
    sc, _ = build_mixed(seed)
    arrays = sc.export_arrays()
    rays = wl.eye_rays_host(wl.camera((0.3, 0.9, 3.2), width=48, height=36))
    rays = np.concatenate([rays, rays[::5] * np.array([1, 1, 1, 1, 1, 1, 1, -1], np.float32)])
    got, cnt, lim = po.port_trace(arrays, rays, counters=True)
    assert lim == 0 and (got["primId"] != MISS).sum() > 100
    if po.ref_available():
        want = po.ref_trace(arrays, rays)
        assert bit_equal(got, want).all(), hit_summary(got, want)


needs_ref = pytest.mark.skipif(not po.ref_available(), reason="reference build absent (make -C oracle ref)")


def _instance_fields_equal(a, b):
    """Bitwise equality of every instance field the traversal reads."""
    for f in ("boxMin", "boxMax", "geomId", "transform", "transformInv", "transformInvTransposed"):
        assert a[f].tobytes() == b[f].tobytes(), f


@needs_ref
def test_instance_matrices_equal_reference_add_and_update_instance():
    """AddInstance / UpdateInstance store the reference's floats
    (BVH2Common_host.cpp:1264-1335, LiteMath inverse4x4): box, transform,
    inverse and normal matrix bit-equal to the reference's own host code for
    rotations with scales from 1e-3 to 50 and translations up to 1e4."""
    v, t = wl.noisy_sphere(12, seed=9)
    mats = (wl.random_instances(600, seed=5) + wl.random_instances(200, seed=6, scale=(1e-3, 50), trans=1e4)
            + [wl.IDENTITY, wl.similarity(0.5, (1, 2, 3))])
    ref = po.RefScene()
    gr = ref.add_triangles(v, t)
    sc = SceneRT()
    gs = sc.AddGeom_Triangles3f(v, t)
    for m in mats:
        ref.add_instance(gr, m)
        sc.AddInstance(gs, m)
    # UpdateInstance: new transform and inverse; the normal matrix stays in both
    new = wl.random_instances(len(mats), seed=8, scale=(0.01, 10), trans=100)
    for i in range(0, len(mats), 7):
        ref.update_instance(i, new[i])
        sc.UpdateInstance(i, new[i])
    ref.commit()
    sc.CommitScene(host_only=True)
    _instance_fields_equal(sc.export_arrays()["instanceData"], ref.export()["instanceData"])


def _interior_rays(n, seed, lo=-5.0, hi=5.0):
    """Seeded rays from points inside the instance cloud in uniform directions."""
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, size=(n, 3))
    r[:, 3] = 1e-4
    r[:, 4:7] = d
    r[:, 7] = 1e9
    return r


@needs_ref
def test_instanced_scene_built_through_product_matches_reference_build():
    """The two-level workload (three noisy-sphere meshes, two frame octrees,
    256 random instances; reduced sizes) assembled through the product's API
    and through the reference's own AddGeom_* / AddInstance / CommitScene:
    every eye ray and every ray from inside the instance cloud gets the same
    hit, bit for bit (the product's SAH tree and the reference's tree differ;
    nearest hits do not depend on them here)."""
    kw = dict(mesh_tris=(2000, 8000, 20000), octree_depth=6, n_instances=256)
    sc = SceneRT()
    wl.build_instanced(sc, **kw)
    sc.CommitScene(host_only=True)
    rb = RefBuilder()
    wl.build_instanced(rb, **kw)
    ref = rb.CommitScene()
    _instance_fields_equal(sc.export_arrays()["instanceData"], ref.export()["instanceData"])
    rays = np.concatenate([wl.eye_rays_host(wl.camera(wl.INSTANCED_EYE, width=256, height=256)),
                           _interior_rays(65536, seed=21)])
    got = po.port_trace(sc.export_arrays(), rays)
    want = ref.trace(rays, threads=os.cpu_count())
    assert (got["primId"] != MISS).sum() > 8000
    assert bit_equal(got, want).all(), hit_summary(got, want)


@needs_ref
@pytest.mark.parametrize("seed", [0, 1])
def test_mixed_scene_built_through_product_matches_reference_build(seed):
    """A mesh, an SBS, a frame octree and an SVS under random instances,
    assembled by both hosts: hits within the specification's tolerance of the
    reference's build (bit-identical apart from near ties)."""
    sc, _ = build_mixed(seed, n_inst=12)
    ref, _ = build_mixed(seed, n_inst=12, sc=RefBuilder())
    _instance_fields_equal(sc.export_arrays()["instanceData"], ref.export()["instanceData"])
    rays = np.concatenate([wl.eye_rays_host(wl.camera((0.3, 0.9, 3.2), width=96, height=72)),
                           _interior_rays(20000, seed=30 + seed, lo=-1.5, hi=1.5)])
    got = po.port_trace(sc.export_arrays(), rays)
    want = ref.trace(rays, threads=os.cpu_count())
    assert (got["primId"] != MISS).sum() > 5000
    rep = assert_within_spec(got, want, what="mixed scene")
    assert rep["bit_identical"] >= len(rays) - rep["ties"]


@needs_ref
def test_triangle_hits_independent_of_builder():
    """Nearest triangle hits do not depend on the tree: the product builder
    and the reference builder give the same answers on a mesh."""
    v, t = wl.noisy_sphere(40, seed=3)
    rays = wl.eye_rays_host(wl.camera((0, 0, 3), width=64, height=64))
    ref = po.RefScene()
    ref.add_instance(ref.add_triangles(v, t), wl.IDENTITY)
    ref.commit()
    want = ref.trace(rays)
    sc = SceneRT()
    sc.AddInstance(sc.AddGeom_Triangles3f(v, t), wl.IDENTITY)
    sc.CommitScene(host_only=True)
    got = po.port_trace(sc.export_arrays(), rays)
    assert bit_equal(got, want).all(), hit_summary(got, want)


def _upload_error(arrays):
    sc = SceneRT()
    with pytest.raises(LrtError) as e:
        sc.upload_arrays(arrays)
    return e.value


def test_upload_validation_rejects_malformed_arrays():
    sc, _ = build_mixed()
    good = sc.export_arrays()

    bad = {k: v.copy() for k, v in good.items()}
    bad["nodesTLAS"]["leftOffset"][0] = LEAF | (1 << 28) | 999
    assert _upload_error(bad).status == 2

    bad = {k: v.copy() for k, v in good.items()}
    bad["nodesTLAS"]["escapeIndex"][1] = 0
    assert _upload_error(bad).status == 2

    bad = {k: v.copy() for k, v in good.items()}
    pairs = bad["allNodePairs"]
    inner = np.nonzero((pairs["left"]["leftOffset"] & LEAF) == 0)[0]
    pairs["left"]["leftOffset"][inner[1]] = 0        # points back at the root pair: a cycle
    assert _upload_error(bad).status == 2

    bad = {k: v.copy() for k, v in good.items()}
    bad["sdfSBSData"] = bad["sdfSBSData"][:-100]
    assert _upload_error(bad).status == 2

    bad = {k: v.copy() for k, v in good.items()}
    bad["instanceData"]["geomId"][0] = 77
    err = _upload_error(bad)
    assert err.status == 2 and "geometry 77" in str(err)


def test_unsupported_presets_are_reported():
    from graphic_lab_task_b200 import default_preset
    sc = SceneRT(preset=default_preset())  # ANALYTIC node intersection, VERTEX normals
    assert sc.GetPreset().sdf_node_intersect == 1


def test_update_instance_host_semantics():
    """UpdateInstance (BVH2Common_host.cpp:1303-1335): new transform, inverse
    and box; the normal matrix stays unless asked for, as in the reference;
    the arrays equal a scene built with the new transform from the start
    (normal matrix refreshed); bad ids and singular matrices are refused."""
    sc, _ = build_mixed(seed=3)
    mats = wl.random_instances(8, seed=33, scale=(0.3, 0.8), trans=1.2)
    before = sc.export_arrays()["instanceData"].copy()
    sc.UpdateInstance(2, mats[2])
    sc.CommitScene(host_only=True)
    after = sc.export_arrays()["instanceData"]
    assert np.array_equal(after[2]["transform"], np.asarray(mats[2], np.float32))
    assert np.array_equal(after[2]["transformInvTransposed"], before[2]["transformInvTransposed"])
    assert not np.array_equal(after[2]["transformInv"], before[2]["transformInv"])
    sc.UpdateInstance(2, mats[2], update_normal_matrix=True)
    sc.UpdateInstance(5, mats[5], update_normal_matrix=True)
    sc.CommitScene(host_only=True)
    # the same scene built with the final transforms from the start
    sph = wl.spheres(12, seed=203)
    fresh = SceneRT()
    v, t = wl.noisy_sphere(20, seed=3)
    gm = fresh.AddGeom_Triangles3f(v, t)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    gb = fresh.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    go = fresh.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 4))
    gs = fresh.AddGeom_SdfSVS(wl.svs_from_spheres(sph, 4))
    orig = wl.random_instances(8, seed=3, scale=(0.3, 0.8), trans=1.2)
    for i, m in enumerate(orig):
        fresh.AddInstance([gm, gb, go, gs][i % 4], mats[i] if i in (2, 5) else m)
    fresh.CommitScene(host_only=True)
    a, b = sc.export_arrays(), fresh.export_arrays()
    for k in ("instanceData", "nodesTLAS"):
        assert a[k].tobytes() == b[k].tobytes(), k
    with pytest.raises(LrtError):
        sc.UpdateInstance(8, mats[0])
    with pytest.raises(LrtError):
        sc.UpdateInstance(0, np.zeros(16, np.float32))


def _write(path, *chunks):
    with open(path, "wb") as f:
        for c in chunks:
            f.write(np.ascontiguousarray(c).tobytes())


def test_sdf_model_files_load_like_the_arrays(tmp_path):
    """The file adders read the reference's model formats
    (sdf/simple/sdf_simple.cpp): the arrays equal those of the in-memory
    adders, an SBS file without the float trailer (the older format) loads
    with its quantised values, and truncated files are refused."""
    sph = wl.spheres(10, seed=31)
    oct_nodes = wl.frame_octree_from_spheres(sph, 4)
    svs = wl.svs_from_spheres(sph, 4)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    u32 = lambda x: np.array([x], np.uint32)  # noqa: E731
    _write(tmp_path / "o.bin", u32(len(oct_nodes)), oct_nodes)
    _write(tmp_path / "s.bin", u32(len(svs)), svs)
    _write(tmp_path / "b.bin", hdr, u32(len(nodes)), nodes, u32(len(vals)), vals, u32(len(vf)), vf)
    a, b = SceneRT(), SceneRT()
    for sc, from_file in ((a, True), (b, False)):
        if from_file:
            g = [sc.AddGeom_SdfFile("frame_octree", tmp_path / "o.bin"), sc.AddGeom_SdfFile("svs", tmp_path / "s.bin"),
                 sc.AddGeom_SdfFile("sbs", tmp_path / "b.bin")]
        else:
            g = [sc.AddGeom_SdfFrameOctree(oct_nodes), sc.AddGeom_SdfSVS(svs), sc.AddGeom_SdfSBS(hdr, nodes, vals, vf)]
        for i, m in enumerate(wl.random_instances(6, seed=5, scale=(0.3, 0.7), trans=1.0)):
            sc.AddInstance(g[i % 3], m)
        sc.CommitScene(host_only=True)
    xa, xb = a.export_arrays(), b.export_arrays()
    for k in xa:
        assert xa[k].tobytes() == xb[k].tobytes(), k
    # the older SBS format: no float-count trailer; a DX (quantised) layout needs no floats
    dx = hdr.copy()
    dx["aux_data"] = 0x01000000  # SDF_SBS_NODE_LAYOUT_DX
    dx["bytes_per_value"] = 4
    _write(tmp_path / "old.bin", dx, u32(len(nodes)), nodes, u32(len(vals)), vals)
    c = SceneRT()
    c.AddGeom_SdfFile("sbs", tmp_path / "old.bin")
    # truncated files
    _write(tmp_path / "t.bin", u32(len(svs) + 5), svs)
    with pytest.raises(LrtError):
        SceneRT().AddGeom_SdfFile("svs", tmp_path / "t.bin")
    _write(tmp_path / "t2.bin", hdr, u32(len(nodes)), nodes, u32(len(vals) + 1), vals)
    with pytest.raises(LrtError):
        SceneRT().AddGeom_SdfFile("sbs", tmp_path / "t2.bin")
    with pytest.raises(LrtError):
        SceneRT().AddGeom_SdfFile("frame_octree", tmp_path / "missing.bin")


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the error without a CUDA device")
def test_device_build_without_device_is_an_error():
    """BUILD_LOW builds the tree on the CUDA device; without one the adder
    fails with LRT_ERR_CUDA and leaves the scene as it was."""
    from graphic_lab_task_b200 import BUILD_LOW
    sc = SceneRT()
    v, t = wl.noisy_sphere(8)
    with pytest.raises(LrtError) as e:
        sc.AddGeom_Triangles3f(v, t, flags=BUILD_LOW)
    assert e.value.status == 4 and "BUILD_LOW" in str(e.value)
    with pytest.raises(LrtError) as e:
        sc.AddGeom_AABB(0, np.array([[0, 0, 0, 1, 1, 1, 1, 1]], np.float32), flags=BUILD_LOW)
    assert e.value.status == 4
    g = sc.AddGeom_Triangles3f(v, t)
    assert g == 0
    sc.AddInstance(g, wl.IDENTITY)
    sc.AddInstance(g, wl.IDENTITY)
    with pytest.raises(LrtError) as e:
        sc.CommitScene(options=BUILD_LOW, host_only=True)
    assert e.value.status == 4
    sc.CommitScene(host_only=True)
    a = sc.export_arrays()
    check_blas_layout(a, 0)
    assert len(a["geomData"]) == 1 and len(a["vertPos"]) == len(v)

"""Shared helpers of the tests: golden fixtures and hit comparison."""
import glob
import os

import numpy as np

from graphic_lab_task_b200._abi import ARRAY_FIELDS, HIT_DTYPE, parity_preset

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MISS = 0xFFFFFFFF


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    arrays = {}
    for field, dt in ARRAY_FIELDS:
        raw = z["arr_" + field]
        if dt.subdtype is not None:  # uint2 / float4 fields
            base, shape = dt.subdtype
            arrays[field] = raw.view(base).reshape((-1,) + shape)
        else:
            arrays[field] = raw.view(dt) if raw.size else np.zeros(0, dt)
    preset = parity_preset()
    p = z["preset"]
    (preset.render_mode, preset.sdf_node_intersect, preset.normal_mode, preset.ray_gen_mode,
     preset.interpolation_mode, preset.representation_mode, preset.spp, preset.fixed_lod) = [int(x) for x in p]
    hits = z["hits"].reshape(-1).view(HIT_DTYPE)
    return arrays, z["rays"], hits, preset


def bit_equal(a, b):
    """Per-ray bitwise equality of two hit arrays."""
    return (a.view(np.uint8).reshape(len(a), 32) == b.view(np.uint8).reshape(len(b), 32)).all(axis=1)


def hit_summary(got, want):
    same = bit_equal(got, want)
    bad = np.nonzero(~same)[0]
    return "%d/%d bit-identical; first mismatches %s" % (same.sum(), len(same), [
        (int(i), tuple(got[i].tolist()), tuple(want[i].tolist())) for i in bad[:3]])


def decode_normal(e):
    """decode_normal (utils/raytracing/render_common.h:257-266), vectorised."""
    e = np.asarray(e, np.float64)
    v = np.stack([e[:, 0], e[:, 1], 1.0 - np.abs(e[:, 0]) - np.abs(e[:, 1])], axis=1)
    neg = v[:, 2] < 0
    vx = v[neg, 0].copy()
    v[neg, 0] = (1.0 - np.abs(v[neg, 1])) * np.where(vx >= 0, 1.0, -1.0)
    v[neg, 1] = (1.0 - np.abs(vx)) * np.where(v[neg, 1] >= 0, 1.0, -1.0)
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def tolerance_report(got, want, rays=None):
    """Compares with the hot-path tolerances: ids exact, t within 1e-5
    relative, decoded normals within 1e-4.  Rays whose hit status or ids
    differ are returned separately (near ties / silhouettes)."""
    hg, hw = got["primId"] != MISS, want["primId"] != MISS
    ids = (got["primId"] == want["primId"]) & (got["instId"] == want["instId"]) & (got["geomId"] == want["geomId"])
    both = hg & hw & ids
    rel_t = np.abs(got["t"][both].astype(np.float64) - want["t"][both]) / np.maximum(np.abs(want["t"][both]), 1e-30)
    ng = decode_normal(got["coords"][both][:, 2:4])
    nw = decode_normal(want["coords"][both][:, 2:4])
    dn = np.abs(ng - nw).max(axis=1) if len(ng) else np.zeros(0)
    return {"id_mismatch": int((~ids).sum()), "max_rel_t": float(rel_t.max()) if len(rel_t) else 0.0,
            "max_normal_err": float(dn.max()) if len(dn) else 0.0, "t_fail": int((rel_t > 1e-5).sum()),
            "n_fail": int((dn > 1e-4).sum()), "mismatch_idx": np.nonzero(~ids)[0]}


def assert_within_spec(got, want, max_tie_frac=1e-4, what="", tree_ref=None, max_tree_frac=1e-6):
    """The hot path's acceptance rule against the reference's own build:
    ids (primId, instId, geomId) bit-exact except on rays whose two nearest
    hits lie within 1e-5 relative t (here: the two answers name different
    primitives at t values within 1e-5 of each other, so the ray has two hits
    that close), t within 1e-5 relative where the ids agree, decoded normals
    within 1e-4 where the ids agree.  Hit/miss disagreements are failures.
    At most `max_tie_frac` of the rays may be near ties.

    Different trees (the product's builder against the reference's) can also
    change an SDF answer by more than 1e-5: the first SDF leaf hit ends a
    BLAS traversal (BVH2Common.cpp:3234-3237, 3310), so which leaf of an
    octree answers depends on the traversal order.  With `tree_ref` (a
    function of ray indices returning the reference code's hits on the
    product's own arrays) such rays pass if the reference, given the
    product's tree, returns the product's hit bit for bit; at most
    `max_tree_frac` of the rays (at least one) may be of this kind."""
    hg, hw = got["primId"] != MISS, want["primId"] != MISS
    assert np.array_equal(hg, hw), "%s: %d rays hit in one and miss in the other" % (what, int((hg != hw).sum()))
    ids = (got["primId"] == want["primId"]) & (got["instId"] == want["instId"]) & (got["geomId"] == want["geomId"])
    rel = np.zeros(len(got))
    rel[hg] = np.abs(got["t"][hg].astype(np.float64) - want["t"][hg]) / np.maximum(np.abs(want["t"][hg]), 1e-30)
    same = hg & ids
    assert (rel[same] <= 1e-5).all(), "%s: %d hits with equal ids outside 1e-5 relative t (max %.3g)" % (
        what, int((rel[same] > 1e-5).sum()), rel[same].max())
    ties = hg & ~ids & (rel <= 1e-5)
    tree = np.nonzero(hg & ~ids & (rel > 1e-5))[0]
    assert ties.sum() <= max(1, max_tie_frac * len(got)), "%s: %d id mismatches (near ties) of %d rays" % (
        what, int(ties.sum()), len(got))
    if len(tree):
        assert tree_ref is not None, "%s: %d rays with other hits more than 1e-5 apart in t (max %.3g)" % (
            what, len(tree), rel[tree].max())
        assert len(tree) <= max(1, max_tree_frac * len(got)), "%s: %d tree-order differences" % (what, len(tree))
        again = tree_ref(tree)
        assert bit_equal(again, got[tree]).all(), "%s: the reference on the product's arrays disagrees on %s" % (
            what, tree[~bit_equal(again, got[tree])][:5])
    rep = tolerance_report(got, want)
    assert rep["n_fail"] == 0, "%s: %d normals outside 1e-4 (max %.3g)" % (what, rep["n_fail"], rep["max_normal_err"])
    rep["ties"] = int(ties.sum())
    rep["tree_order"] = int(len(tree))
    rep["bit_identical"] = int(bit_equal(got, want).sum())
    return rep


class RefBuilder:
    """The reference's own scene assembly (pyoracle.RefScene: BVHRT
    AddGeom_* / AddInstance / CommitScene compiled from its sources) behind
    the method names of SceneRT, so that one workload generator builds the
    same scene through both."""

    def __init__(self, fast=False):
        import pyoracle
        self.ref = pyoracle.RefScene(fast=fast)

    def AddGeom_Triangles3f(self, verts, tris):
        return self.ref.add_triangles(verts, tris)

    def AddGeom_SdfFrameOctree(self, nodes):
        return self.ref.add_frame_octree(nodes)

    def AddGeom_SdfSVS(self, nodes):
        return self.ref.add_svs(nodes)

    def AddGeom_SdfSBS(self, header, nodes, values, values_f=None):
        return self.ref.add_sbs(header, nodes, values, values_f)

    def AddInstance(self, geom, matrix):
        return self.ref.add_instance(geom, matrix)

    def CommitScene(self):
        self.ref.commit()
        return self.ref


LEAF = 0x80000000


def check_blas_layout(arrays, geom, base=None):
    """The fat-pair BLAS of geometry `geom` (its pairs from `base`, by
    default its geomData bvhOffset) is a depth-first pre-order tree (every
    inner pointer points forward, no pair reached twice) whose leaves name
    each entry of its leaf table once, Pack(id, 1); returns the leaf ids in
    traversal order."""
    pairs, gd, se = arrays["allNodePairs"], arrays["geomData"], arrays["startEnd"]
    base = int(gd["bvhOffset"][geom]) if base is None else base
    a0, a1 = int(se[geom][0]), int(se[geom][1])
    seen, ids, stack = set(), [], [0]
    while stack:
        k = stack.pop()
        assert k not in seen
        seen.add(k)
        for side in ("left", "right"):
            lo = int(pairs[base + k][side]["leftOffset"])
            if lo & LEAF:
                if lo != 0xFFFFFFFF and lo != LEAF:
                    assert (lo & 0x0FFFFFFF) < a1 - a0
                    assert (lo >> 28) & 7 == 1      # Pack(id, 1)
                    ids.append(lo & 0x0FFFFFFF)
            else:
                assert lo > k                       # depth-first pre-order
                stack.append(lo)
    assert sorted(ids) == list(range(a1 - a0))
    return ids


def check_tlas_layout(nodes, n_inst):
    """The escape-index TLAS: aligned sibling pairs, the left one escaping
    to its sibling and the right one to its parent's escape, each instance
    in exactly one leaf, and every inner box containing its children."""
    assert nodes[0]["escapeIndex"] == 1 and nodes[1]["escapeIndex"] == 0xFFFFFFFE
    leaves = []
    stack = [(0, 0xFFFFFFFE)]
    while stack:
        a, esc = stack.pop()
        assert nodes[a]["escapeIndex"] == a + 1 and nodes[a + 1]["escapeIndex"] == esc
        for j in (0, 1):
            n = nodes[a + j]
            lo = int(n["leftOffset"])
            if lo & LEAF:
                leaves.append(lo & 0x0FFFFFFF)
            else:
                assert lo > a
                for c in (lo, lo + 1):
                    assert np.all(nodes[c]["boxMin"] >= n["boxMin"]) and np.all(nodes[c]["boxMax"] <= n["boxMax"])
                stack.append((lo, int(n["escapeIndex"])))
    assert sorted(leaves) == list(range(n_inst))


def _spread3_6(x):
    x = x & 0x3F
    x = (x | (x << 8)) & 0x0000F00F
    x = (x | (x << 4)) & 0x000C30C3
    x = (x | (x << 2)) & 0x00249249
    return x


def bounce_coherence_keys(bounce, instance_data):
    """The sort key of lrt_generate_bounce_rays_sorted, restated in numpy
    float32 from its definition in include/lrt_b200.h: direction cell of a
    4x4x4 grid over [-1, 1]^3 above the 6-bit-per-axis Morton code of the
    origin in the union of the instances' world boxes."""
    bmin = instance_data["boxMin"][:, :3].astype(np.float32)
    bmax = instance_data["boxMax"][:, :3].astype(np.float32)
    lo = np.zeros(3, np.float32)
    scale = np.zeros(3, np.float32)
    for k in range(3):
        ok = bmin[:, k] <= bmax[:, k]
        if not ok.any():
            continue
        lo[k] = bmin[ok, k].min()
        ext = np.float32(bmax[ok, k].max() - lo[k])
        if ext > 0 and np.isfinite(ext):
            scale[k] = np.float32(64) / ext
    o = bounce[:, 0:3].astype(np.float32)
    d = bounce[:, 4:7].astype(np.float32)
    with np.errstate(invalid="ignore"):
        f = (o - lo) * scale
        q = np.where(~(f > 0), 0, np.where(f >= 63, 63, np.nan_to_num(f).astype(np.int64)))
        g = (d + np.float32(1)) * np.float32(2)
        c = np.where(~(g > 0), 0, np.where(g >= 3, 3, np.nan_to_num(g).astype(np.int64)))
    cell = (c[:, 0] << 4) | (c[:, 1] << 2) | c[:, 2]
    morton = (_spread3_6(q[:, 0]) << 2) | (_spread3_6(q[:, 1]) << 1) | _spread3_6(q[:, 2])
    return np.minimum((cell << 18) | morton, (1 << 24) - 2).astype(np.int64)

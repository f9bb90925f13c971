"""Generates the golden vectors in tests/golden/*.npz from the reference itself.

Run here (where the reference sources exist), after ``make -C oracle ref``:

    python tests/golden/make_golden.py

Every scene is assembled by the reference's own host code (BVHRT::AddGeom_*,
AddInstance, CommitScene in MultiRenderer/BVH2Common_host.cpp, with the
Embree build-API shim of oracle/ref) and every hit comes from the reference's
BVHRT::RayQuery_NearestHit (MultiRenderer/BVH2Common.cpp:3322-3392) built with
-ffp-contract=off (oracle/_ref/liblrt_ref.so).  Each file stores the flattened
BVHRT arrays, the preset, the rays and the reference hits, so the oracle
restatement (CPU tests) and the CUDA kernels (GPU tests, uploaded through
lrt_scene_upload) can be checked against them bit for bit.

Scenes: hand-made single-triangle and one-brick cases (axis-parallel rays,
rays inside boxes, the 0.01 leaf bias, any-hit rays), a small noisy-sphere
mesh, a small sphere-union SBS, an instanced frame-octree/SVS/mesh scene,
and three SDF models saved in the reference repository (a frame octree from
scenes/06_engine_scenes/framed_octree/ and spatial crops of
saves/test_10_svs.bin and saves/test_10_sbs.bin, read with a length check
because test_10_sbs.bin predates the values_f_count trailer).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyoracle as po  # noqa: E402
from graphic_lab_task_b200 import workloads as wl  # noqa: E402
from graphic_lab_task_b200._abi import (FRAME_OCTREE_NODE_DTYPE, SBS_HEADER_DTYPE, SBS_NODE_DTYPE,  # noqa: E402
                                        SVS_NODE_DTYPE, parity_preset)

REF = po.reference_src()


def preset_array(p):
    return np.array([p.render_mode, p.sdf_node_intersect, p.normal_mode, p.ray_gen_mode, p.interpolation_mode,
                     p.representation_mode, p.spp, p.fixed_lod], np.uint32)


def save(name, ref, rays, note):
    arrays = ref.export()
    hits = ref.trace(rays)
    out = {"rays": rays.astype(np.float32), "hits": hits.view(np.uint8).reshape(len(hits), 32),
           "preset": preset_array(ref.preset), "note": np.array(note)}
    for k, v in arrays.items():
        out["arr_" + k] = v.view(np.uint8).reshape(-1) if v.size else np.zeros(0, np.uint8)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    nh = int(np.sum(hits["primId"] != 0xFFFFFFFF))
    print("%-22s rays %6d hits %6d  %7.1f KB" % (name, len(rays), nh, os.path.getsize(path) / 1024))


def camera_rays(eye, w, h, tnear=1e-4, center=(0, 0, 0)):
    return wl.eye_rays_host(wl.camera(eye, center=center, width=w, height=h, tnear=tnear))


def random_rays(n, seed, center=(0, 0, 0), spread=1.0, origin_radius=3.0):
    rng = np.random.default_rng(seed)
    o = rng.normal(size=(n, 3))
    o = o / np.linalg.norm(o, axis=1, keepdims=True) * origin_radius
    target = np.asarray(center) + rng.uniform(-spread, spread, size=(n, 3))
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = o
    r[:, 3] = 1e-4
    r[:, 4:7] = d
    r[:, 7] = 1e9
    return r


def any_hit(rays):
    r = rays.copy()
    r[:, 7] = -r[:, 7]
    return r


def hand_triangle():
    ref = po.RefScene()
    v = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    g = ref.add_triangles(v, np.array([0, 1, 2], np.uint32))
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    R = []

    def ray(o, d, tn=1e-4, tf=1e9):
        R.append([o[0], o[1], o[2], tn, d[0], d[1], d[2], tf])

    ray((0.25, 0.25, 1), (0, 0, -1))              # straight down, zero x/y direction components
    ray((0.25, 0.25, -1), (0, 0, 1))              # from behind
    ray((0.25, 0.25, 0.005), (0, 0, -1))          # hit at t=0.005 < SDF_BIAS 0.01: rejected
    ray((0.25, 0.25, 0.02), (0, 0, -1))           # hit at t=0.02: accepted
    ray((0.25, 0.25, 1), (0, 0, -1), 1e-4, 0.5)   # tfar before the triangle
    ray((0.25, 0.25, 1), (0, 0, -1), 1e-4, -1e9)  # any-hit (negative tfar)
    ray((0.5, 0.5, 1), (0, 0, -1))                # on the hypotenuse u+v=1
    ray((1.0, 0.0, 1), (0, 0, -1))                # on a vertex
    ray((-1e-7, 0.5, 1), (0, 0, -1))              # just outside an edge (1e-6 tolerance)
    ray((2, 2, 1), (0, 0, -1))                    # clear miss
    ray((-1, 0.25, 0), (1, 0, 0))                 # in the triangle's plane
    ray((0.2, 0.2, 0.5), (0.1, 0.1, -1))          # oblique
    for a in np.linspace(0, 2 * np.pi, 20, endpoint=False):
        ray((0.3, 0.3, 2), (0.3 * np.cos(a), 0.3 * np.sin(a), -1))
    rays = np.array(R, np.float32)
    d = rays[:, 4:7]
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    save("hand_triangle", ref, rays, "single triangle, hand rays")


def hand_brick():
    # one 4^3 brick over [-1,1]^3 holding a tilted plane, DX layout, 4 bytes per value
    bs, pad = 4, 0
    v = bs + 2 * pad + 1
    hdr = np.zeros(1, SBS_HEADER_DTYPE)
    hdr["brick_size"], hdr["brick_pad"], hdr["bytes_per_value"], hdr["aux_data"] = bs, pad, 4, 1 << 24
    node = np.zeros(1, SBS_NODE_DTYPE)
    node["pos_xy"], node["pos_z_lod_size"], node["data_offset"] = 0, 1, 0
    d_max = np.float32(1.73205081) * np.float32(2.0)
    vals = np.zeros(v ** 3, np.uint32)
    n = np.array([0.3, 0.5, 0.8])
    n /= np.linalg.norm(n)
    for x in range(v):
        for y in range(v):
            for z in range(v):
                p = -1 + 2 * np.array([x, y, z]) / bs
                dist = float(np.dot(p, n)) - 0.1
                q = (dist + d_max) / (2 * d_max) * 4294967295.0
                vals[(x * v + y) * v + z] = np.uint32(min(max(round(q), 0), 4294967295))
    ref = po.RefScene()
    g = ref.add_sbs(hdr, node, vals)
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    rays = camera_rays((2.0, 2.5, 3.0), 24, 24)
    save("hand_brick", ref, np.concatenate([rays, any_hit(rays[::7])]), "one DX brick, tilted plane")


def mesh_small():
    v, t = wl.noisy_sphere(24, seed=7)
    ref = po.RefScene()
    g = ref.add_triangles(v, t)
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    rays = np.concatenate([camera_rays((0, 0, 3), 48, 48), random_rays(512, 11), any_hit(random_rays(128, 12))])
    save("mesh_small", ref, rays, "noisy UV sphere, 1104 triangles")


def sbs_small():
    sph = wl.spheres(16, seed=5)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    ref = po.RefScene()
    g = ref.add_sbs(hdr, nodes, vals, vf)
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    rays = np.concatenate([camera_rays((0, 0, 3), 64, 48), random_rays(512, 13), any_hit(random_rays(128, 14))])
    save("sbs_small", ref, rays, "16-sphere SBS, virtual 32^3, 4^3 bricks, indexed fp32")


def instanced_mix():
    sph = wl.spheres(16, seed=6)
    oct_nodes = wl.frame_octree_from_spheres(sph, 4)
    svs = wl.svs_from_spheres(sph, 4)
    v, t = wl.noisy_sphere(12, seed=8)
    ref = po.RefScene()
    go = ref.add_frame_octree(oct_nodes)
    gs = ref.add_svs(svs)
    gm = ref.add_triangles(v, t)
    for i, m in enumerate(wl.random_instances(9, seed=9, scale=(0.4, 0.9), trans=1.5)):
        ref.add_instance([go, gs, gm][i % 3], m)
    ref.commit()
    rays = np.concatenate([camera_rays((0, 0, 4), 48, 48), random_rays(512, 15, spread=2.0, origin_radius=4.0),
                           any_hit(random_rays(256, 16, spread=2.0, origin_radius=4.0))])
    save("instanced_mix", ref, rays, "frame octree + SVS + mesh, 9 instances")


def node_solvers():
    """The same frame-octree + SVS + SBS scene under the ANALYTIC (the
    reference's default), NEWTON and IT node solvers of
    LocalSurfaceIntersection (BVH2Common.cpp:392-618)."""
    sph = wl.spheres(16, seed=6)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=32, brick_size=4, brick_pad=1)
    for mode, name in ((1, "solver_analytic"), (2, "solver_newton"), (4, "solver_it")):
        p = parity_preset()
        p.sdf_node_intersect = mode
        ref = po.RefScene(preset=p)
        gb = ref.add_sbs(hdr, nodes, vals, vf)
        go = ref.add_frame_octree(wl.frame_octree_from_spheres(sph, 4))
        gs = ref.add_svs(wl.svs_from_spheres(sph, 4))
        for i, m in enumerate(wl.random_instances(9, seed=21, scale=(0.4, 0.9), trans=1.2)):
            ref.add_instance([gb, go, gs][i % 3], m)
        ref.commit()
        rays = np.concatenate([camera_rays((0, 0, 4), 48, 48), random_rays(1024, 22, spread=2.0, origin_radius=4.0),
                               any_hit(random_rays(128, 23, spread=2.0, origin_radius=4.0))])
        save(name, ref, rays, "SBS + frame octree + SVS, 9 instances, sdf_node_intersect %d" % mode)


def read_u32(f):
    return int(np.frombuffer(f.read(4), np.uint32)[0])


def ref_frame_octree():
    path = os.path.join(REF, "scenes/06_engine_scenes/framed_octree/sdf_frame_octree_0.bin")
    with open(path, "rb") as f:
        n = read_u32(f)
        nodes = np.frombuffer(f.read(n * FRAME_OCTREE_NODE_DTYPE.itemsize), FRAME_OCTREE_NODE_DTYPE).copy()
    ref = po.RefScene()
    g = ref.add_frame_octree(nodes)
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    rays = np.concatenate([camera_rays((0.3, 0.5, 2.5), 48, 48), random_rays(512, 17), any_hit(random_rays(64, 18))])
    save("ref_frame_octree", ref, rays, "reference model sdf_frame_octree_0.bin (%d nodes)" % n)


def crop_lod_nodes(nodes, frac=0.5):
    px = nodes["pos_xy"] >> 16
    sz = nodes["pos_z_lod_size"] & 0xFFFF
    return nodes[px < frac * sz]


def ref_svs():
    path = os.path.join(REF, "saves/test_10_svs.bin")
    with open(path, "rb") as f:
        n = read_u32(f)
        nodes = np.frombuffer(f.read(n * SVS_NODE_DTYPE.itemsize), SVS_NODE_DTYPE).copy()
    nodes = crop_lod_nodes(nodes, 0.35)
    ref = po.RefScene()
    g = ref.add_svs(nodes)
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    rays = np.concatenate([camera_rays((-2.0, 0.8, 2.0), 48, 48, center=(-0.65, 0, 0)),
                           random_rays(256, 19, center=(-0.65, 0, 0), spread=0.5)])
    save("ref_svs_crop", ref, rays, "reference model test_10_svs.bin, nodes with x < 0.35 (%d)" % len(nodes))


def ref_sbs():
    path = os.path.join(REF, "saves/test_10_sbs.bin")
    size = os.path.getsize(path)
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(16), SBS_HEADER_DTYPE).copy()
        n = read_u32(f)
        nodes = np.frombuffer(f.read(n * 16), SBS_NODE_DTYPE).copy()
        cnt = read_u32(f)
        values = np.frombuffer(f.read(cnt * 4), np.uint32).copy()
        rest = size - f.tell()
        values_f = np.zeros(0, np.float32)
        if rest >= 4:  # files written after values_f_count was added
            cf = read_u32(f)
            values_f = np.frombuffer(f.read(cf * 4), np.float32).copy()
    keep = crop_lod_nodes(nodes, 0.35)
    # compact the kept bricks' words
    bs, pad, bpv = int(hdr["brick_size"][0]), int(hdr["brick_pad"][0]), int(hdr["bytes_per_value"][0])
    v3 = (bs + 2 * pad + 1) ** 3
    words = (v3 * bpv + 3) // 4
    new_vals = np.concatenate([values[o:o + words] for o in keep["data_offset"]])
    keep["data_offset"] = np.arange(len(keep), dtype=np.uint32) * words
    ref = po.RefScene()
    g = ref.add_sbs(hdr, keep, new_vals, values_f if len(values_f) else None)
    ref.add_instance(g, wl.IDENTITY)
    ref.commit()
    rays = np.concatenate([camera_rays((-2.0, 0.8, 2.0), 48, 48, center=(-0.65, 0, 0)),
                           random_rays(256, 20, center=(-0.65, 0, 0), spread=0.5)])
    save("ref_sbs_crop", ref, rays, "reference model test_10_sbs.bin (DX, %d B/value), bricks with x < 0.35 (%d)"
         % (bpv, len(keep)))


def main():
    if not po.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    hand_triangle()
    hand_brick()
    mesh_small()
    sbs_small()
    instanced_mix()
    node_solvers()
    if os.path.isdir(REF):
        ref_frame_octree()
        ref_svs()
        ref_sbs()


if __name__ == "__main__":
    main()

"""Seeded synthetic workloads of the ray-query benchmark.

Five configurations (the reference publishes no benchmark inputs, so these
seeded generators stand in for them, with the shapes the specification
names):

0. a noisy UV sphere of ~200k triangles, one 256x256 pinhole camera;
1. a sparse brick set (8^3 bricks, 1 voxel border, fp32 distances through the
   indexed layout) of the union of 64 seeded spheres sampled on a virtual
   512^3 grid, 1920x1080 camera;
2. 1024 instances of three noisy spheres (50k/200k/500k triangles) and two
   frame-octree SDF objects (depth 8), 4096^2 primary rays plus one
   cosine-weighted bounce per hit;
3. the configuration-1 scene seen by 64 cameras on a radius-3 sphere with
   log-uniform square resolutions in [128, 2048];
4. an SBS at virtual 256^3 rendered from 16 views of 512x512 (adjoint form).

Geometry comes from liblrt_b200.so (include/lrt_workloads.h); cameras and
host eye rays are computed here.  ``eye_rays_host`` evaluates
MultiRenderer::initEyeRay in float32 in the same operation order as the
device generator, so the two agree bit for bit.
"""
import ctypes as C
import math

import numpy as np

from ._abi import (FRAME_OCTREE_NODE_DTYPE, SBS_HEADER_DTYPE, SBS_NODE_DTYPE, SVS_NODE_DTYPE, Camera)
from .lrt import check, lib

F = np.float32


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------
def noisy_sphere(segments=317, radius=1.0, amplitude=0.05, seed=0):
    """UV sphere with 2*s*(s-1) triangles (s=317 -> 200,344), vertices pushed
    along the normal by seeded value noise of the given amplitude."""
    L = lib()
    nv, nt = C.c_uint64(), C.c_uint64()
    check(L.lrt_wl_noisy_sphere(segments, radius, amplitude, seed, None, None, C.byref(nv), C.byref(nt)))
    verts = np.zeros((nv.value, 3), np.float32)
    tris = np.zeros((nt.value, 3), np.uint32)
    check(L.lrt_wl_noisy_sphere(segments, radius, amplitude, seed, verts.ctypes.data, tris.ctypes.data, C.byref(nv),
                                C.byref(nt)))
    return verts, tris


def segments_for_triangles(ntris):
    """Smallest UV-sphere segment count with at least `ntris` triangles."""
    s = max(3, int(math.ceil((1 + math.sqrt(1 + 2 * ntris)) / 2)))
    while 2 * s * (s - 1) < ntris:
        s += 1
    return s


def spheres(n=64, c=0.8, rmin=0.05, rmax=0.3, seed=1):
    out = np.zeros((n, 4), np.float32)
    check(lib().lrt_wl_spheres(n, c, rmin, rmax, seed, out.ctypes.data))
    return out


def sbs_from_spheres(sph, grid_res=512, brick_size=8, brick_pad=1):
    """(header, nodes, values, values_f) of an ID32F_IRGB32F sparse brick set."""
    L = lib()
    s = np.ascontiguousarray(sph, np.float32)
    nn, nv, nf = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(L.lrt_wl_sbs_from_spheres(s.ctypes.data, len(s), grid_res, brick_size, brick_pad, None, None, None, None,
                                    C.byref(nn), C.byref(nv), C.byref(nf)))
    header = np.zeros(1, SBS_HEADER_DTYPE)
    nodes = np.zeros(nn.value, SBS_NODE_DTYPE)
    values = np.zeros(nv.value, np.uint32)
    values_f = np.zeros(nf.value, np.float32)
    check(L.lrt_wl_sbs_from_spheres(s.ctypes.data, len(s), grid_res, brick_size, brick_pad, header.ctypes.data,
                                    nodes.ctypes.data, values.ctypes.data, values_f.ctypes.data, C.byref(nn),
                                    C.byref(nv), C.byref(nf)))
    return header, nodes, values, values_f


def frame_octree_from_spheres(sph, max_depth=8):
    L = lib()
    s = np.ascontiguousarray(sph, np.float32)
    n = C.c_uint64()
    check(L.lrt_wl_frame_octree_from_spheres(s.ctypes.data, len(s), max_depth, None, C.byref(n)))
    nodes = np.zeros(n.value, FRAME_OCTREE_NODE_DTYPE)
    check(L.lrt_wl_frame_octree_from_spheres(s.ctypes.data, len(s), max_depth, nodes.ctypes.data, C.byref(n)))
    return nodes


def svs_from_spheres(sph, lod=6):
    L = lib()
    s = np.ascontiguousarray(sph, np.float32)
    n = C.c_uint64()
    check(L.lrt_wl_svs_from_spheres(s.ctypes.data, len(s), lod, None, C.byref(n)))
    nodes = np.zeros(n.value, SVS_NODE_DTYPE)
    check(L.lrt_wl_svs_from_spheres(s.ctypes.data, len(s), lod, nodes.ctypes.data, C.byref(n)))
    return nodes


# ---------------------------------------------------------------------------
# transforms and cameras (column-major 4x4 as LiteMath float4x4)
# ---------------------------------------------------------------------------
def col_major(m):
    """row/column indexed 4x4 (m[r][c]) -> 16 floats, element (r,c) at [c*4+r]."""
    return np.ascontiguousarray(np.asarray(m, np.float64).T.reshape(16), dtype=np.float32)


IDENTITY = col_major(np.eye(4))


def similarity(scale, translation):
    """Column-major matrix of a uniform scale followed by a translation."""
    m = np.eye(4)
    m[:3, :3] *= scale
    m[:3, 3] = translation
    return col_major(m)


def look_at(eye, center, up):
    """LiteMath lookAt (LiteMath.h:3315-3340): the world-to-view matrix."""
    eye, center, up = (np.asarray(v, np.float64) for v in (eye, center, up))
    z = eye - center
    z /= np.linalg.norm(z)
    x = np.cross(up, z)
    y = np.cross(z, x)
    x /= np.linalg.norm(x)
    y /= np.linalg.norm(y)
    m = np.eye(4)
    m[0, :3], m[1, :3], m[2, :3] = x, y, z
    m[0, 3], m[1, 3], m[2, 3] = -x @ eye, -y @ eye, -z @ eye
    return m


def perspective(fovy_deg, aspect, znear, zfar):
    """LiteMath perspectiveMatrix (LiteMath.h:3342-3362)."""
    ymax = znear * math.tan(fovy_deg * math.pi / 360.0)
    xmax = ymax * aspect
    m = np.zeros((4, 4))
    m[0, 0] = 2 * znear / (2 * xmax)
    m[1, 1] = 2 * znear / (2 * ymax)
    m[2, 2] = (-zfar - znear) / (zfar - znear)
    m[3, 2] = -1.0
    m[2, 3] = (-2 * znear * zfar) / (zfar - znear)
    return m


def camera(eye, center=(0, 0, 0), up=(0, 1, 0), fovy=60.0, width=256, height=256, tnear=1e-4, tfar=1e9):
    """lrt_camera for MultiRenderer::initEyeRay (zNear 0.01, zFar 100 as in
    MultiRenderer_host.cpp:1078)."""
    z = np.asarray(eye, np.float64) - np.asarray(center, np.float64)
    if abs(np.dot(z / np.linalg.norm(z), up)) > 0.999:
        up = (1, 0, 0)
    view = look_at(eye, center, up)
    proj = perspective(fovy, width / height, 0.01, 100.0)
    cam = Camera()
    pinv = col_major(np.linalg.inv(proj))
    vinv = col_major(np.linalg.inv(view))
    for i in range(16):
        cam.proj_inv[i] = float(pinv[i])
        cam.world_view_inv[i] = float(vinv[i])
    cam.width, cam.height, cam.tnear, cam.tfar = width, height, tnear, tfar
    return cam


def sample_offset(sample, spp, ray_gen_mode=0):
    """initEyeRay's position of sample `sample` of `spp` in the pixel
    (MultiRenderer.cpp:162-166, first frame): a regular sqrt(spp) grid, or
    the first Hamilton point for RAY_GEN_MODE_RANDOM."""
    if ray_gen_mode == 1:
        return F(0.5), F(0.333333)
    q = int(math.sqrt(spp))
    inv = F(1.0) / F(q)
    return inv * F(sample // q + 0.5), inv * F(sample % q + 0.5)


def eye_rays_host(cam, dx=0.5, dy=0.5):
    """(H*W, 8) float32 rays in row-major pixel order through the points
    (x + dx, y + dy) of the pixels; the float32 evaluation order matches
    lrt::eye_ray (csrc/lrt_math.h)."""
    W, H = cam.width, cam.height
    P = np.array(cam.proj_inv[:], np.float32)
    M = np.array(cam.world_view_inv[:], np.float32)
    idx = np.arange(W * H, dtype=np.int64)
    x = (idx % W).astype(np.float32)
    y = (idx // W).astype(np.float32)
    with np.errstate(all="ignore"):
        fx = (x + F(dx)) / F(W)
        fy = (y + F(dy)) / F(H)
        px = F(2.0) * fx - F(1.0)
        py = F(-2.0) * fy + F(1.0)
        q = [px * P[i] + py * P[4 + i] + F(1.0) * P[8 + i] + F(1.0) * P[12 + i] for i in range(4)]
        d = [q[0] / q[3], q[1] / q[3], q[2] / q[3]]
        inv = F(1.0) / np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        d = [c * inv for c in d]
        zero = F(0.0)
        pos = [zero * M[i] + zero * M[4 + i] + zero * M[8 + i] + F(1.0) * M[12 + i] for i in range(3)]
        p2in = [zero + F(100.0) * c for c in d]
        pos2 = [p2in[0] * M[i] + p2in[1] * M[4 + i] + p2in[2] * M[8 + i] + F(1.0) * M[12 + i] for i in range(3)]
        diff = [pos2[i] - pos[i] for i in range(3)]
        inv = F(1.0) / np.sqrt(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2])
        d = [c * inv for c in diff]
    rays = np.zeros((W * H, 8), np.float32)
    for i in range(3):
        rays[:, i] = pos[i]
        rays[:, 4 + i] = d[i]
    rays[:, 3] = F(cam.tnear)
    rays[:, 7] = F(cam.tfar)
    return rays


def sphere_cameras(n, radius=3.0, res_min=128, res_max=2048, seed=3, fixed_res=None):
    """n cameras on a sphere looking at the origin: seeded uniform directions,
    square resolutions log-uniform in [res_min, res_max] (or fixed_res)."""
    rng = np.random.default_rng(seed)
    cams = []
    for _ in range(n):
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        r = fixed_res or int(round(math.exp(rng.uniform(math.log(res_min), math.log(res_max)))))
        cams.append(camera(radius * v, width=r, height=r))
    return cams


LIGHT = (0.577, 0.577, 0.577)

# Incoherent two-level workload: eye far enough out to see the instance cloud
INSTANCED_EYE = (0.0, 0.0, 12.0)


def build_instanced(scene, mesh_tris=(50000, 200000, 500000), octree_depth=8, n_instances=1024, seed=2,
                    n_spheres=64, sphere_seed=1):
    """Adds three noisy-sphere meshes (about `mesh_tris` triangles) and two
    frame-octree SDF objects of the sphere union (depth `octree_depth`) to
    `scene`, then `n_instances` instances with random similarity transforms
    (uniform rotation, scale U[0.05, 0.2], translation U[-5, 5]^3), instance i
    of geometry i % 5.  The two octree geometries hold the same octree: the
    reference keeps one global origNodes array, overwritten by every
    AddGeom_SdfFrameOctree (BVH2Common_host.cpp:531), so distinct octrees
    would make the first one read the second one's boxes."""
    geoms = []
    for n in mesh_tris:
        v, t = noisy_sphere(segments_for_triangles(n), seed=n)
        geoms.append(scene.AddGeom_Triangles3f(v, t))
    nodes = frame_octree_from_spheres(spheres(n_spheres, seed=sphere_seed), octree_depth)
    geoms.append(scene.AddGeom_SdfFrameOctree(nodes))
    geoms.append(scene.AddGeom_SdfFrameOctree(nodes))
    for i, m in enumerate(random_instances(n_instances, seed=seed)):
        scene.AddInstance(geoms[i % len(geoms)], m)
    return geoms


def adjoint_workload(grid_res=256, views=16, res=512, noise=0.01, seed=4, n_spheres=64, sphere_seed=1):
    """Differentiable-render workload: the sphere-union SBS at `grid_res`^3,
    `views` cameras of res x res on a radius-3 sphere, and target values =
    the distances plus N(0, noise) per voxel value (palette untouched).
    Returns (header, nodes, values, values_f, target_values_f, cameras, rays)."""
    sph = spheres(n_spheres, seed=sphere_seed)
    hdr, nodes, vals, vf = sbs_from_spheres(sph, grid_res=grid_res)
    rng = np.random.default_rng(seed)
    target = vf.copy()
    first = 3 * n_spheres  # the palette precedes the distances
    target[first:] += rng.normal(0.0, noise, size=len(vf) - first).astype(np.float32)
    cams = sphere_cameras(views, radius=3.0, seed=seed + 1, fixed_res=res)
    rays = np.concatenate([eye_rays_host(c) for c in cams])
    return hdr, nodes, vals, vf, target, cams, rays


def random_instances(n, seed=2, scale=(0.05, 0.2), trans=5.0):
    """n column-major transforms: uniform rotation (random unit quaternion),
    uniform scale in `scale`, translation U[-trans, trans]^3."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        s = rng.uniform(*scale)
        m = np.eye(4)
        m[:3, :3] = R * s
        m[:3, 3] = rng.uniform(-trans, trans, size=3)
        out.append(col_major(m))
    return out

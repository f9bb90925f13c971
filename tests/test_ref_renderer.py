"""The oracle's restatements of the renderer around the ray query, pinned to
the reference's own MultiRenderer compiled from its sources (oracle/_ref,
oracle/ref/render_harness.cpp) on the same scene (the reference's own build):

* initEyeRay (MultiRenderer.cpp:142-183): every sample position of the
  sqrt(spp) grid and RAY_GEN_MODE_RANDOM's Hamilton point;
* Render (MultiRenderer.cpp:14-60) in every render mode the fused render
  implements: kernel1D_FillGbuffer, ResolveCommon / ResolveDebug /
  ResolveOutline (MultiRenderer_resolve.cpp), several samples, the
  transparency path, and kernel1D_Tonemap;
* kernel1D_FillGbufferWithTransparency with AnyHit (MultiRenderer.cpp:
  204-246): the composited float4 and the last hit of every pixel.

All bit for bit.  The GPU kernels are compared with the same restatements in
tests/test_gpu_render.py, so these tests close the chain GPU = restatement =
reference.  No GPU needed.  Image sizes are multiples of 8, the renderer's
tile padding (for other widths it resolves pixels with other pixels' rays)."""
import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import (LIGHT_AMBIENT, LIGHT_DIRECT, LIGHT_DTYPE, LIGHT_POINT, MATERIAL_COLORED,
                                   parity_preset, workloads as wl)
from helpers import RefBuilder, bit_equal

pytestmark = pytest.mark.skipif(not po.ref_available(), reason="reference build absent (make -C oracle ref)")

BG = (0.1, 0.2, 0.3, 1.0)
EYE = (0.5, 0.7, 3.5)
# the render modes of lrt_render_rgba8 (core/render_settings.h:61-88) without
# textures, shadows or data channels; 13 OUTLINE_PRIM
RENDER_MODES = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 16, 17, 18, 19, 20, 21, 22, 24, 25]


def _lights():
    lt = np.zeros(3, LIGHT_DTYPE)
    d = np.array([0.4, 0.8, 0.45], np.float32)
    lt[0] = (d / np.linalg.norm(d), LIGHT_DIRECT, (0.9, 0.85, 0.7), 0)
    lt[1] = ((1.5, 2.0, 2.5), LIGHT_POINT, (4.0, 3.0, 2.0), 0)
    lt[2] = ((0, 0, 0), LIGHT_AMBIENT, (0.05, 0.06, 0.08), 0)
    return lt


@pytest.fixture(scope="module")
def mixed():
    """A mesh, a frame octree, an SVS and an SBS under 40 random instances,
    assembled by the reference's own host code; the renderer's mesh copy of
    the triangles (MultiRenderer::add_mesh_internal)."""
    sph = wl.spheres(32, seed=4)
    rb = RefBuilder()
    v, t = wl.noisy_sphere(60, seed=2)
    gm = rb.AddGeom_Triangles3f(v, t)
    go = rb.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 6))
    gs = rb.AddGeom_SdfSVS(wl.svs_from_spheres(sph, 6))
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64)
    gb = rb.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    for i, m in enumerate(wl.random_instances(40, seed=7, scale=(0.1, 0.4), trans=1.5)):
        rb.AddInstance([gm, go, gs, gb][i % 4], m)
    ref = rb.CommitScene()
    return {"ref": ref, "arrays": ref.export(), "mesh": (gm, v, t)}


def _renderer(s, cam, preset, materials=None):
    r = po.RefRenderer(s["ref"])
    gm, v, t = s["mesh"]
    r.add_mesh(gm, v, t)
    r.set_camera(cam)
    r.set_lights(_lights())
    r.set_background(BG)
    r.set_preset(preset)
    if materials is not None:
        r.set_materials(*materials)
    return r


def _camera(w, h):
    # initEyeRay's own interval: tNear 1e-9, tFar 1e9 with the cutting plane off
    return wl.camera(EYE, width=w, height=h, tnear=1e-9, tfar=1e9)


def _materials(seed, opaque=True):
    from test_oracle import transparency_tables
    mats, ids, offs = transparency_tables(4, seed=seed)
    mats["type"] = MATERIAL_COLORED
    if opaque:
        mats["base_color"][:, 3] = 1.0
    mats["metallic"] = np.linspace(0, 1, len(mats))
    mats["roughness"] = np.linspace(0.2, 0.9, len(mats))
    return mats, ids, offs


@pytest.mark.parametrize("spp,ray_gen", [(1, 0), (4, 0), (16, 0), (4, 1)])
def test_eye_rays_equal_reference_init_eye_ray(mixed, spp, ray_gen):
    cam = _camera(96, 64)
    p = parity_preset()
    p.spp, p.ray_gen_mode = spp, ray_gen
    r = _renderer(mixed, cam, p)
    for k in range(min(spp, 4)):
        dx, dy = wl.sample_offset(k, spp, ray_gen)
        want = r.eye_rays(cam.width, cam.height, k)
        got = wl.eye_rays_host(cam, dx, dy)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (spp, ray_gen, k)
    r.close()


@pytest.mark.parametrize("mode", RENDER_MODES)
def test_render_modes_equal_reference_render(mixed, mode):
    cam = _camera(160, 120)
    p = parity_preset()
    p.render_mode = mode
    mats = _materials(11)
    r = _renderer(mixed, cam, p, mats)
    want = r.render(cam.width, cam.height)
    got = po.port_render_rgba8(mixed["arrays"], wl.eye_rays_host(cam), _lights(), BG, preset=p, materials=mats[0],
                               mat_ids=mats[1], mat_offsets=mats[2])
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    assert len(np.unique(want)) >= 2  # hits and background in view
    r.close()


@pytest.mark.parametrize("mode,spp,ray_gen,transparent", [(1, 4, 0, False), (17, 4, 0, False), (12, 2, 1, False),
                                                           (17, 1, 0, True), (16, 4, 0, True), (18, 4, 0, True),
                                                           (21, 4, 0, True)])
def test_samples_and_transparency_equal_reference_render(mixed, mode, spp, ray_gen, transparent):
    cam = _camera(96, 64)
    p = parity_preset()
    p.render_mode, p.spp, p.ray_gen_mode = mode, spp, ray_gen
    mats = _materials(12, opaque=not transparent)
    r = _renderer(mixed, cam, p, mats)
    want = r.render(cam.width, cam.height)
    offsets = [wl.sample_offset(k, spp, ray_gen) for k in range(spp)]
    sample_rays = np.stack([wl.eye_rays_host(cam, dx, dy) for dx, dy in offsets])
    got = po.port_render_rgba8_samples(mixed["arrays"], sample_rays, sample_rays[0], _lights(), BG, p,
                                       materials=mats[0], mat_ids=mats[1], mat_offsets=mats[2],
                                       transparency=transparent)
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    r.close()


@pytest.mark.parametrize("spp", [1, 4])
def test_outline_border_equals_reference_render(mixed, spp):
    cam = _camera(96, 64)
    p = parity_preset()
    p.render_mode, p.spp = 14, spp
    r = _renderer(mixed, cam, p)
    want = r.render(cam.width, cam.height)
    offsets = [wl.sample_offset(k, spp, 0) for k in range(spp)]
    sample_rays = np.stack([wl.eye_rays_host(cam, dx, dy) for dx, dy in offsets])
    got = po.port_render_outline_border(mixed["arrays"], sample_rays, sample_rays[0], cam.width, cam.height,
                                        _lights(), BG, p)
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    outline = (255 << 24) | (51 << 16) | (51 << 8) | 51
    assert (want == outline).sum() > 20
    r.close()


def test_fill_gbuffer_transparency_equals_reference_any_hit(mixed):
    from test_oracle import transparency_tables
    a = mixed["arrays"]
    mats, ids, offs = transparency_tables(len(a["geomData"]), seed=3)
    cam = _camera(200, 152)
    r = _renderer(mixed, cam, parity_preset(), (mats, ids, offs))
    want_t, want_h = r.fill_transparency(cam.width, cam.height)
    got_t, got_h, capped = po.port_fill_gbuffer_transparency(a, wl.eye_rays_host(cam), mats, ids, offs,
                                                             np.array(BG, np.float32))
    assert capped == 0
    same = (got_t.view(np.uint32) == want_t.view(np.uint32)).all(axis=1) & bit_equal(got_h, want_h)
    assert same.all(), "%d of %d pixels differ" % ((~same).sum(), len(same))
    assert (want_t[:, 3] < 0.99).sum() > 500
    r.close()


def _textures(seed=5):
    """Slot 0 as a new MultiRenderer holds it (16x16 of (0, 1, 1, 1)), then a
    seeded random 37x23 image and a 64x64 checker."""
    rng = np.random.default_rng(seed)
    default = np.zeros((16, 16, 4), np.float32)
    default[:] = (0, 1, 1, 1)
    noise = rng.uniform(0, 1, size=(23, 37, 4)).astype(np.float32)
    yy, xx = np.mgrid[0:64, 0:64]
    checker = np.zeros((64, 64, 4), np.float32)
    checker[..., 0] = ((xx // 8 + yy // 8) % 2).astype(np.float32)
    checker[..., 1] = 0.3
    checker[..., 2] = xx / 63.0
    checker[..., 3] = 1
    return [default, noise, checker]


def mesh_texcoords(verts):
    """Seeded-free spherical texture coordinates of a mesh around the origin,
    beyond [0, 1] in places (the sampler clamps)."""
    v = np.asarray(verts, np.float64)
    u = np.arctan2(v[:, 2], v[:, 0]) / (2 * np.pi) + 0.5
    w = np.arccos(np.clip(v[:, 1] / np.linalg.norm(v, axis=1), -1, 1)) / np.pi
    return np.stack([1.3 * u - 0.15, w], axis=1).astype(np.float32)


def _textured_materials():
    from graphic_lab_task_b200 import MATERIAL_TEXTURED
    mats, ids, offs = _materials(13)
    mats["type"][1::2] = MATERIAL_TEXTURED
    mats["texId"] = np.arange(len(mats)) % 3
    return mats, ids, offs


@pytest.mark.parametrize("mode", [15, 16, 17, 18, 21, 11])
def test_textured_materials_equal_reference_render(mixed, mode):
    """TEXTURED materials in DIFFUSE, LAMBERT, PHONG and PBR (PBR_NO_TEX with
    a textured material 0) and the TEX_COORDS mode: the reference's
    bilinear / clamp sampling at loadNormalTcFromGbuffer's coordinates
    (barycentric blend of the mesh's per-vertex coordinates, the hit's coords
    for SDF leaves), restated bit for bit."""
    from graphic_lab_task_b200 import MATERIAL_TEXTURED
    cam = _camera(160, 120)
    p = parity_preset()
    p.render_mode = mode
    mats, ids, offs = _textured_materials()
    if mode == 11:
        mats["type"][0] = MATERIAL_TEXTURED
        mats["texId"][0] = 2
    gm, v, t = mixed["mesh"]
    tc = mesh_texcoords(v)
    r = po.RefRenderer(mixed["ref"])
    r.add_mesh(gm, v, t, tc)
    texs = _textures()
    assert [r.add_texture(x) for x in texs[1:]] == [1, 2]
    r.set_camera(cam)
    r.set_lights(_lights())
    r.set_background(BG)
    r.set_preset(p)
    r.set_materials(mats, ids, offs)
    want = r.render(cam.width, cam.height)
    a = mixed["arrays"]
    vert_tc = np.zeros((len(a["vertPos"]), 2), np.float32)
    off = int(a["geomData"]["offset"][gm][1])
    vert_tc[off:off + len(v)] = tc
    po.port_set_textures(texs, vert_tc)
    got = po.port_render_rgba8(a, wl.eye_rays_host(cam), _lights(), BG, preset=p, materials=mats, mat_ids=ids,
                               mat_offsets=offs)
    po.port_set_textures(None)
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    assert len(np.unique(want)) > 50
    r.close()


def test_textured_samples_and_transparency_equal_reference_render(mixed):
    """Four samples per pixel, LAMBERT, a transparent COLORED material beside
    the TEXTURED ones: the AnyHit G-buffer (textured layers opaque black) and
    the resolve's texture samples, blended as ResolveTransparency does."""
    cam = _camera(96, 64)
    p = parity_preset()
    p.render_mode, p.spp = 17, 4
    mats, ids, offs = _textured_materials()
    mats["base_color"][0, 3] = 0.4
    gm, v, t = mixed["mesh"]
    tc = mesh_texcoords(v)
    r = po.RefRenderer(mixed["ref"])
    r.add_mesh(gm, v, t, tc)
    texs = _textures()
    for x in texs[1:]:
        r.add_texture(x)
    r.set_camera(cam)
    r.set_lights(_lights())
    r.set_background(BG)
    r.set_preset(p)
    r.set_materials(mats, ids, offs)
    want = r.render(cam.width, cam.height)
    a = mixed["arrays"]
    vert_tc = np.zeros((len(a["vertPos"]), 2), np.float32)
    off = int(a["geomData"]["offset"][gm][1])
    vert_tc[off:off + len(v)] = tc
    po.port_set_textures(texs, vert_tc)
    sample_rays = np.stack([wl.eye_rays_host(cam, *wl.sample_offset(k, 4, 0)) for k in range(4)])
    got = po.port_render_rgba8_samples(a, sample_rays, sample_rays[0], _lights(), BG, p, materials=mats, mat_ids=ids,
                                       mat_offsets=offs, transparency=True)
    po.port_set_textures(None)
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    r.close()

"""Fused camera render (lrt_render_rgba8): eye rays, nearest hit, the
resolve of the preset's render mode (LAMBERT_NO_TEX with direct, point and
ambient lights, and the other modes without textures, shadows or PBR) and the
tonemap in one launch, bit-identical to the oracle's restatement of
MultiRenderer's Render on the same scene arrays; and the transparency loop."""
import numpy as np
import pytest

import pyoracle as po
from graphic_lab_task_b200 import (HIT_DTYPE, LIGHT_AMBIENT, LIGHT_DIRECT, LIGHT_DTYPE, LIGHT_POINT, LrtError,
                                   SceneRT, parity_preset, workloads as wl)
from helpers import bit_equal

pytestmark = pytest.mark.gpu


def _lights():
    lt = np.zeros(3, LIGHT_DTYPE)
    d = np.array([0.4, 0.8, 0.45], np.float32)
    lt[0] = (d / np.linalg.norm(d), LIGHT_DIRECT, (0.9, 0.85, 0.7), 0)
    lt[1] = ((1.5, 2.0, 2.5), LIGHT_POINT, (4.0, 3.0, 2.0), 0)
    lt[2] = ((0, 0, 0), LIGHT_AMBIENT, (0.05, 0.06, 0.08), 0)
    return lt


def _mixed_scene():
    sph = wl.spheres(32, seed=4)
    sc = SceneRT()
    v, t = wl.noisy_sphere(60, seed=2)
    gm = sc.AddGeom_Triangles3f(v, t)
    go = sc.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 6))
    gs = sc.AddGeom_SdfSVS(wl.svs_from_spheres(sph, 6))
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64)
    gb = sc.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    for i, m in enumerate(wl.random_instances(40, seed=7, scale=(0.1, 0.4), trans=1.5)):
        sc.AddInstance([gm, go, gs, gb][i % 4], m)
    sc.CommitScene()
    return sc


@pytest.mark.parametrize("size", [(200, 150), (256, 128)])
def test_render_rgba8_matches_oracle(cuda, size):
    torch = cuda
    sc = _mixed_scene()
    cam = wl.camera((0.5, 0.7, 3.5), width=size[0], height=size[1])
    bg = (0.1, 0.2, 0.3, 1.0)
    img = torch.zeros(size[0] * size[1], dtype=torch.int32, device="cuda")
    sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
    sc.sync()
    got = img.cpu().numpy().view(np.uint32)
    want = po.port_render_rgba8(sc.export_arrays(), wl.eye_rays_host(cam), _lights(), bg)
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    for _ in range(3):  # the tile schedule the first launches measured reorders the later ones
        img.zero_()
        sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
        sc.sync()
        assert np.array_equal(img.cpu().numpy().view(np.uint32), want)
    bgpx = (255 << 24) | (int(255 * 0.3) << 16) | (int(255 * 0.2) << 8) | int(255 * 0.1)
    assert 0.05 < (got != bgpx).mean() < 0.95  # both hits and background in view
    assert len(np.unique(got)) > 100


def test_render_rgba8_refusals(cuda):
    torch = cuda
    sc = _mixed_scene()
    cam = wl.camera((0.5, 0.7, 3.5), width=16, height=16)
    img = torch.zeros(256, dtype=torch.int32, device="cuda")
    many = np.zeros(17, LIGHT_DTYPE)
    with pytest.raises(LrtError) as e:
        sc.render_rgba8(cam, many, (0, 0, 0, 1), img.data_ptr())
    assert e.value.status == 1
    p = parity_preset()
    p.render_mode = 23  # CHANNEL
    sc.SetPreset(p)
    with pytest.raises(LrtError) as e:
        sc.render_rgba8(cam, _lights(), (0, 0, 0, 1), img.data_ptr())
    assert e.value.status == 6 and "render_mode 23" in str(e.value)
    p.render_mode = 11  # PBR_NO_TEX shades with material 0
    sc.SetPreset(p)
    with pytest.raises(LrtError) as e:
        sc.render_rgba8(cam, _lights(), (0, 0, 0, 1), img.data_ptr())
    assert e.value.status == 1 and "material 0" in str(e.value)
    from graphic_lab_task_b200 import MATERIAL_TEXTURED
    from test_oracle import transparency_tables
    for mode in (16, 17, 18, 21, 22):  # materials needed
        p.render_mode = mode
        sc.SetPreset(p)
        with pytest.raises(LrtError) as e:
            sc.render_rgba8(cam, _lights(), (0, 0, 0, 1), img.data_ptr())
        assert e.value.status == 1 and "material range" in str(e.value)
    mats, ids, offs = transparency_tables(4)  # has transparent and textured materials, no texture is set
    sc.set_materials(mats, ids, offs)
    p.render_mode = 17
    sc.SetPreset(p)
    with pytest.raises(LrtError) as e:
        sc.render_rgba8(cam, _lights(), (0, 0, 0, 1), img.data_ptr())
    assert e.value.status == 1 and "texture" in str(e.value)
    mats["base_color"][:, 3] = 1.0  # opaque, but one is textured and no texture is set
    sc.set_materials(mats, ids, offs)
    with pytest.raises(LrtError) as e:
        sc.render_rgba8(cam, _lights(), (0, 0, 0, 1), img.data_ptr())
    assert e.value.status == 1 and "texture" in str(e.value)
    assert (mats["type"] == MATERIAL_TEXTURED).any()


# the render modes of ResolveCommon / kernel1D_ResolveDebug without textures,
# shadows or PBR (core/render_settings.h:61-88)
RENDER_MODES = [0, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 16, 17, 18, 19, 20, 21, 22, 24, 25]


@pytest.mark.parametrize("mode", RENDER_MODES)
def test_render_modes_match_oracle(cuda, mode):
    """lrt_render_rgba8 in every implemented render mode equals the oracle's
    restatement of Render pixel for pixel (NORMAL, Phong and PBR within one
    8-bit step: their pow is CUDA's on the device)."""
    torch = cuda
    from graphic_lab_task_b200 import MATERIAL_COLORED
    from test_oracle import transparency_tables
    sc = _mixed_scene()
    mats, ids, offs = transparency_tables(4, seed=11)
    mats["type"] = MATERIAL_COLORED
    mats["base_color"][:, 3] = 1.0
    mats["metallic"] = np.linspace(0, 1, len(mats))
    mats["roughness"] = np.linspace(0.2, 0.9, len(mats))
    sc.set_materials(mats, ids, offs)
    p = parity_preset()
    p.render_mode = mode
    sc.SetPreset(p)
    cam = wl.camera((0.5, 0.7, 3.5), width=160, height=120)
    bg = (0.1, 0.2, 0.3, 1.0)
    img = torch.zeros(cam.width * cam.height, dtype=torch.int32, device="cuda")
    sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
    sc.sync()
    got = img.cpu().numpy().view(np.uint32)
    want = po.port_render_rgba8(sc.export_arrays(), wl.eye_rays_host(cam), _lights(), bg, preset=p, materials=mats,
                                mat_ids=ids, mat_offsets=offs)
    if mode in (8, 11, 12, 18, 21):
        d = np.abs(got.view(np.uint8).astype(int) - want.view(np.uint8).astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 0.01
    else:
        assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    bgpx = (255 << 24) | (int(255 * 0.3) << 16) | (int(255 * 0.2) << 8) | int(255 * 0.1)
    assert 0.05 < (got != bgpx).mean()  # hits in view


@pytest.mark.parametrize("mode,spp,ray_gen,transparent", [(1, 4, 0, False), (17, 4, 0, False), (12, 2, 1, False),
                                                           (17, 1, 0, True), (16, 4, 0, True), (18, 4, 0, True),
                                                           (21, 4, 0, True)])
def test_render_samples_and_transparency_match_oracle(cuda, mode, spp, ray_gen, transparent):
    """Several samples per pixel (initEyeRay's sqrt(spp) grid, or the first
    Hamilton point for RAY_GEN_MODE_RANDOM; the resolve uses sample 0's ray,
    the colours are averaged) and, with a transparent material in DIFFUSE /
    LAMBERT / PHONG, the AnyHit G-buffer blended into the resolved colour:
    bit-identical to the oracle (Phong within one 8-bit step)."""
    torch = cuda
    from graphic_lab_task_b200 import MATERIAL_COLORED
    from test_oracle import transparency_tables
    sc = _mixed_scene()
    mats, ids, offs = transparency_tables(4, seed=12)
    mats["type"] = MATERIAL_COLORED
    if not transparent:
        mats["base_color"][:, 3] = 1.0
    assert transparent == bool((mats["base_color"][:, 3] < 1).any())
    sc.set_materials(mats, ids, offs)
    p = parity_preset()
    p.render_mode, p.spp, p.ray_gen_mode = mode, spp, ray_gen
    sc.SetPreset(p)
    cam = wl.camera((0.5, 0.7, 3.5), width=96, height=64)
    bg = (0.1, 0.2, 0.3, 1.0)
    img = torch.zeros(cam.width * cam.height, dtype=torch.int32, device="cuda")
    sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
    sc.sync()
    got = img.cpu().numpy().view(np.uint32)
    offsets = [wl.sample_offset(k, spp, ray_gen) for k in range(spp)]
    sample_rays = np.stack([wl.eye_rays_host(cam, dx, dy) for dx, dy in offsets])
    want = po.port_render_rgba8_samples(sc.export_arrays(), sample_rays, sample_rays[0], _lights(), bg, p,
                                        materials=mats, mat_ids=ids, mat_offsets=offs, transparency=transparent)
    if mode in (12, 18, 21):
        d = np.abs(got.view(np.uint8).astype(int) - want.view(np.uint8).astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 0.01
    else:
        assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    if spp > 1 and ray_gen == 0:  # the samples differ: averaging shows at silhouettes
        one = po.port_render_rgba8_samples(sc.export_arrays(), sample_rays[:1], sample_rays[0], _lights(), bg, p,
                                           materials=mats, mat_ids=ids, mat_offsets=offs, transparency=transparent)
        assert (one != want).sum() > 10


@pytest.mark.parametrize("spp,size", [(1, (96, 64)), (4, (96, 64)), (1, (61, 37))],
                         ids=["spp1", "spp4", "ragged"])
def test_render_outline_border_matches_oracle(cuda, spp, size):
    """OUTLINE_BORDER: per sample a G-buffer pass and ResolveOutline's test
    against the four neighbours' t (more than 10 t / width apart: the
    (0.2, 0.2, 0.2) outline colour), summed over the samples; bit-identical to
    the oracle, repeated on the stream's tile schedule."""
    torch = cuda
    sc = _mixed_scene()
    p = parity_preset()
    p.render_mode, p.spp = 14, spp
    sc.SetPreset(p)
    cam = wl.camera((0.5, 0.7, 3.5), width=size[0], height=size[1])
    bg = (0.1, 0.2, 0.3, 1.0)
    offsets = [wl.sample_offset(k, spp, 0) for k in range(spp)]
    sample_rays = np.stack([wl.eye_rays_host(cam, dx, dy) for dx, dy in offsets])
    want = po.port_render_outline_border(sc.export_arrays(), sample_rays, sample_rays[0], cam.width, cam.height,
                                         _lights(), bg, p)
    for _ in range(3):
        img = torch.zeros(cam.width * cam.height, dtype=torch.int32, device="cuda")
        sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
        sc.sync()
        got = img.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    outline = (255 << 24) | (51 << 16) | (51 << 8) | 51  # tonemap of (0.2, 0.2, 0.2, 1)
    if spp == 1:
        assert (got == outline).sum() > 20
    prim = po.port_render_rgba8_samples(sc.export_arrays(), sample_rays, sample_rays[0], _lights(), bg,
                                        _preset_mode(p, 13))
    assert (prim != want).sum() > 20  # the outlines are what OUTLINE_PRIM does not draw


def test_batched_render_equals_per_camera_render(cuda):
    """lrt_batch_render_rgba8 renders every camera of a batch in one launch;
    each image equals lrt_render_rgba8's for that camera."""
    torch = cuda
    from graphic_lab_task_b200.lrt import CameraBatch
    sc = _mixed_scene()
    cams = wl.sphere_cameras(6, radius=3.5, res_min=40, res_max=130, seed=5)
    b = CameraBatch(sc, cams)
    imgs = torch.zeros(b.total_rays, dtype=torch.int32, device="cuda")
    bg = (0.1, 0.2, 0.3, 1.0)
    b.render_rgba8(_lights(), bg, imgs.data_ptr())
    b.sync()
    got = imgs.cpu().numpy().view(np.uint32)
    off = 0
    for c in cams:
        k = c.width * c.height
        one = torch.zeros(k, dtype=torch.int32, device="cuda")
        sc.render_rgba8(c, _lights(), bg, one.data_ptr())
        sc.sync()
        assert np.array_equal(got[off:off + k], one.cpu().numpy().view(np.uint32))
        off += k
    assert len(np.unique(got)) > 100
    b.close()


def test_fill_gbuffer_transparency_matches_oracle(cuda):
    """kernel1D_FillGbufferWithTransparency on the device: the composited
    float4 and the last hit of every pixel are bit-identical to the oracle's
    AnyHit loop."""
    torch = cuda
    from test_oracle import transparency_tables
    sc = _mixed_scene()
    a = sc.export_arrays()
    mats, ids, offs = transparency_tables(len(a["geomData"]), seed=3)
    sc.set_materials(mats, ids, offs)
    cam = wl.camera((0.5, 0.7, 3.5), width=200, height=150)
    bg = np.array([0.1, 0.2, 0.3, 1.0], np.float32)
    n = cam.width * cam.height
    tr = torch.zeros(n * 4, dtype=torch.float32, device="cuda")
    hits = torch.zeros(n * 8, dtype=torch.float32, device="cuda")
    sc.fill_gbuffer_transparency(cam, bg, tr.data_ptr(), hits.data_ptr())
    sc.sync()
    got_t = tr.cpu().numpy().reshape(-1, 4)
    got_h = hits.cpu().numpy().view(HIT_DTYPE).reshape(-1)
    want_t, want_h, capped = po.port_fill_gbuffer_transparency(a, wl.eye_rays_host(cam), mats, ids, offs, bg)
    assert capped == 0
    for k in range(3):  # launches 2 and 3 follow the tile schedule of the earlier ones
        if k:
            tr.zero_()
            hits.zero_()
            sc.fill_gbuffer_transparency(cam, bg, tr.data_ptr(), hits.data_ptr())
            sc.sync()
            got_t = tr.cpu().numpy().reshape(-1, 4)
            got_h = hits.cpu().numpy().view(HIT_DTYPE).reshape(-1)
        same = (got_t.view(np.uint32) == want_t.view(np.uint32)).all(axis=1) & bit_equal(got_h, want_h)
        assert same.all(), "%d of %d pixels differ" % ((~same).sum(), n)
    assert (got_t[:, 3] < 0.99).sum() > 500  # composited layers


def test_fill_gbuffer_transparency_refusals_and_layer_bound(cuda):
    torch = cuda
    from test_oracle import transparency_tables
    sc = _mixed_scene()
    cam = wl.camera((0.5, 0.7, 3.5), width=32, height=32)
    tr = torch.zeros(32 * 32 * 4, dtype=torch.float32, device="cuda")
    hits = torch.zeros(32 * 32 * 8, dtype=torch.float32, device="cuda")
    bg = (0.1, 0.2, 0.3, 1.0)
    with pytest.raises(LrtError) as e:  # no materials for the mesh
        sc.fill_gbuffer_transparency(cam, bg, tr.data_ptr(), hits.data_ptr())
    assert e.value.status == 1 and "material range" in str(e.value)
    mats, ids, offs = transparency_tables(4)
    bad = ids.copy()
    bad[0] = len(mats)
    with pytest.raises(LrtError) as e:
        sc.set_materials(mats, bad, offs)
    assert e.value.status == 1
    with pytest.raises(LrtError) as e:
        sc.set_materials(mats, ids, offs + np.array([0, 1000], np.uint32))
    assert e.value.status == 1
    # a transparent background never brings alpha down: the reference loops
    # forever on rays that miss; here they stop at the layer bound
    sc.set_materials(mats, ids, offs)
    sc.fill_gbuffer_transparency(cam, (0.1, 0.2, 0.3, 0.0), tr.data_ptr(), hits.data_ptr())
    with pytest.raises(LrtError) as e:
        sc.sync()
    assert e.value.status == 5 and "transparency" in str(e.value)
    sc.fill_gbuffer_transparency(cam, bg, tr.data_ptr(), hits.data_ptr())
    sc.sync()


def _preset_mode(p, mode):
    q = parity_preset()
    q.render_mode, q.spp, q.ray_gen_mode = mode, p.spp, p.ray_gen_mode
    return q


def _textured_scene():
    """The mixed scene with spherical texture coordinates on its mesh, the
    textures of tests/test_ref_renderer.py and half the materials TEXTURED."""
    from test_ref_renderer import _textured_materials, _textures, mesh_texcoords
    sph = wl.spheres(32, seed=4)
    sc = SceneRT()
    v, t = wl.noisy_sphere(60, seed=2)
    gm = sc.AddGeom_Triangles3f(v, t)
    go = sc.AddGeom_SdfFrameOctree(wl.frame_octree_from_spheres(sph, 6))
    gs = sc.AddGeom_SdfSVS(wl.svs_from_spheres(sph, 6))
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64)
    gb = sc.AddGeom_SdfSBS(hdr, nodes, vals, vf)
    for i, m in enumerate(wl.random_instances(40, seed=7, scale=(0.1, 0.4), trans=1.5)):
        sc.AddInstance([gm, go, gs, gb][i % 4], m)
    sc.CommitScene()
    tc = mesh_texcoords(v)
    sc.set_texcoords(gm, tc)
    texs = _textures()
    sc.set_textures(texs)
    a = sc.export_arrays()
    vert_tc = np.zeros((len(a["vertPos"]), 2), np.float32)
    off = int(a["geomData"]["offset"][gm][1])
    vert_tc[off:off + len(v)] = tc
    mats, ids, offs = _textured_materials()
    return sc, a, texs, vert_tc, (mats, ids, offs)


@pytest.mark.parametrize("mode", [15, 16, 17, 18, 21, 11])
def test_render_textured_materials_match_oracle(cuda, mode):
    """TEXTURED materials (bilinear, clamped sampling at the hit's texture
    coordinates) in DIFFUSE, LAMBERT, PHONG, PBR and PBR_NO_TEX, and the
    TEX_COORDS mode: the images equal the oracle's restatement, which
    equals the reference's own renderer (tests/test_ref_renderer.py); Phong
    and PBR within one 8-bit step (CUDA's pow)."""
    torch = cuda
    from graphic_lab_task_b200 import MATERIAL_TEXTURED
    sc, a, texs, vert_tc, (mats, ids, offs) = _textured_scene()
    if mode == 11:
        mats["type"][0] = MATERIAL_TEXTURED
        mats["texId"][0] = 2
    sc.set_materials(mats, ids, offs)
    p = parity_preset()
    p.render_mode = mode
    sc.SetPreset(p)
    cam = wl.camera((0.5, 0.7, 3.5), width=160, height=120)
    bg = (0.1, 0.2, 0.3, 1.0)
    img = torch.zeros(cam.width * cam.height, dtype=torch.int32, device="cuda")
    sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
    sc.sync()
    got = img.cpu().numpy().view(np.uint32)
    po.port_set_textures(texs, vert_tc)
    want = po.port_render_rgba8(a, wl.eye_rays_host(cam), _lights(), bg, preset=p, materials=mats, mat_ids=ids,
                                mat_offsets=offs)
    po.port_set_textures(None)
    if mode in (11, 18, 21):
        d = np.abs(got.view(np.uint8).astype(int) - want.view(np.uint8).astype(int))
        assert d.max() <= 1 and (d > 0).mean() < 0.01
    else:
        assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))
    assert len(np.unique(got)) > 50


def test_render_textured_samples_and_transparency_match_oracle(cuda):
    """Four samples per pixel with a transparent COLORED material beside the
    TEXTURED ones (LAMBERT takes the AnyHit path; the resolve samples the
    textures of the last hit's material)."""
    torch = cuda
    sc, a, texs, vert_tc, (mats, ids, offs) = _textured_scene()
    mats["base_color"][0, 3] = 0.4
    sc.set_materials(mats, ids, offs)
    p = parity_preset()
    p.render_mode, p.spp = 17, 4
    sc.SetPreset(p)
    cam = wl.camera((0.5, 0.7, 3.5), width=96, height=64)
    bg = (0.1, 0.2, 0.3, 1.0)
    img = torch.zeros(cam.width * cam.height, dtype=torch.int32, device="cuda")
    sc.render_rgba8(cam, _lights(), bg, img.data_ptr())
    sc.sync()
    got = img.cpu().numpy().view(np.uint32)
    sample_rays = np.stack([wl.eye_rays_host(cam, *wl.sample_offset(k, 4, 0)) for k in range(4)])
    po.port_set_textures(texs, vert_tc)
    want = po.port_render_rgba8_samples(a, sample_rays, sample_rays[0], _lights(), bg, p, materials=mats,
                                        mat_ids=ids, mat_offsets=offs, transparency=True)
    po.port_set_textures(None)
    assert np.array_equal(got, want), "%d of %d pixels differ" % ((got != want).sum(), len(got))


def test_texture_api_refusals(cuda):
    from graphic_lab_task_b200 import MATERIAL_TEXTURED
    sc, a, texs, vert_tc, (mats, ids, offs) = _textured_scene()
    bad = mats.copy()
    bad["type"][0] = MATERIAL_TEXTURED
    bad["texId"][0] = 3  # three textures are set
    sc.set_materials(bad, ids, offs)
    p = parity_preset()
    p.render_mode = 17
    sc.SetPreset(p)
    torch = cuda
    img = torch.zeros(64, dtype=torch.int32, device="cuda")
    with pytest.raises(LrtError) as e:
        sc.render_rgba8(wl.camera((0.5, 0.7, 3.5), width=8, height=8), _lights(), (0, 0, 0, 1), img.data_ptr())
    assert e.value.status == 1 and "texture 3 of 3" in str(e.value)
    with pytest.raises(LrtError) as e:
        sc.set_texcoords(0, np.zeros((5, 2), np.float32))  # not the mesh's vertex count
    assert e.value.status == 1 and "vertices" in str(e.value)
    with pytest.raises(LrtError) as e:
        sc.set_texcoords(1, np.zeros((5, 2), np.float32))  # the frame octree
    assert e.value.status == 1 and "not a triangle mesh" in str(e.value)
    with pytest.raises(LrtError) as e:
        sc.set_textures([np.zeros((0, 4, 4), np.float32)])
    assert e.value.status == 1

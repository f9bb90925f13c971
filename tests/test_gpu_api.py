"""C-ABI behaviour on the GPU: device-pointer traces on several streams,
unsupported presets, alignment checks and the bounded voxel march reporting
LRT_ERR_DEVICE_LIMIT with the context still usable."""
import numpy as np
import pytest

from graphic_lab_task_b200 import LrtError, SceneRT, default_preset, parity_preset, workloads as wl
from helpers import bit_equal, load_golden

pytestmark = pytest.mark.gpu


def _sbs_scene():
    arrays, rays, want, preset = load_golden("sbs_small")
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    return sc, rays, want


def test_device_pointer_traces_on_two_streams(cuda):
    torch = cuda
    sc, rays, want = _sbs_scene()
    R = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    H1 = torch.zeros(len(rays) * 8, dtype=torch.float32, device="cuda")
    H2 = torch.zeros_like(H1)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    for _ in range(3):
        sc.trace_device(R.data_ptr(), H1.data_ptr(), len(rays), stream=s1.cuda_stream)
        sc.trace_device(R.data_ptr(), H2.data_ptr(), len(rays), stream=s2.cuda_stream)
    sc.sync(stream=s1.cuda_stream)
    sc.sync(stream=s2.cuda_stream)
    from graphic_lab_task_b200 import HIT_DTYPE
    for H in (H1, H2):
        got = H.cpu().numpy().view(HIT_DTYPE)
        assert bit_equal(got, want).all()


@pytest.mark.parametrize("memory", ["pinned", "pageable"])
@pytest.mark.parametrize("n", [262144, 300001, 1000003])
def test_host_buffer_traces_equal_device_trace(cuda, n, memory):
    """Host-buffer traces of 262144 rays or more run as a chunked
    copy/trace/copy pipeline over several streams: chunks of 32768 rays for
    the smaller n (the last one ragged for 300001), chunk sizes ramping
    32768 -> 262144 and back for n = 1000003.  Every hit equals the
    single-launch device-pointer trace and the oracle."""
    torch = cuda
    import pyoracle as po
    from graphic_lab_task_b200 import HIT_DTYPE
    sph = wl.spheres(16, seed=3)
    hdr, nodes, vals, vf = wl.sbs_from_spheres(sph, grid_res=64)
    sc = SceneRT()
    sc.AddInstance(sc.AddGeom_SdfSBS(hdr, nodes, vals, vf), wl.IDENTITY)
    sc.CommitScene()
    rays = wl.eye_rays_host(wl.camera((0, 0, 3), width=1000, height=1002))[:n]
    rays = np.ascontiguousarray(rays)
    if memory == "pinned":
        host_rays = torch.from_numpy(rays).pin_memory()
        host_hits = torch.zeros(n * 8, dtype=torch.float32).pin_memory()
        sc.trace_host(host_rays.data_ptr(), host_hits.data_ptr(), n)
        got = host_hits.numpy().view(HIT_DTYPE)
    else:
        got = sc.RayQuery_NearestHitBatch(rays)
    R = torch.from_numpy(rays).cuda()
    H = torch.zeros(n * 8, dtype=torch.float32, device="cuda")
    sc.trace_device(R.data_ptr(), H.data_ptr(), n)
    sc.sync()
    assert bit_equal(got, H.cpu().numpy().view(HIT_DTYPE)).all()
    idx = np.unique(np.linspace(0, n - 1, 4096).astype(np.int64))
    assert bit_equal(got[idx], po.port_trace(sc.export_arrays(), rays[idx])).all()
    assert (got["primId"] != 0xFFFFFFFF).sum() > 1000


def test_misaligned_device_pointer_is_rejected(cuda):
    torch = cuda
    sc, rays, _ = _sbs_scene()
    R = torch.zeros(len(rays) * 8 + 4, dtype=torch.float32, device="cuda")
    H = torch.zeros(len(rays) * 8, dtype=torch.float32, device="cuda")
    with pytest.raises(LrtError) as e:
        sc.trace_device(R.data_ptr() + 4, H.data_ptr(), len(rays))
    assert e.value.status == 1 and "aligned" in str(e.value)


def test_unsupported_preset_is_refused(cuda):
    """The plain trace implements all five node solvers (the reference's
    default preset uses ANALYTIC); the batched, render and adjoint calls
    implement ST and BBOX and refuse the others; a solver id outside 0..4 is
    refused everywhere."""
    torch = cuda
    sc, rays, _ = _sbs_scene()
    sc.SetPreset(default_preset())
    sc.RayQuery_NearestHitBatch(rays[:8])
    R = torch.from_numpy(np.ascontiguousarray(rays[:64])).cuda()
    img = torch.empty(64, dtype=torch.float32, device="cuda")
    with pytest.raises(LrtError) as e:
        sc.render_lambert(R.data_ptr(), 64, wl.LIGHT, img.data_ptr())
    assert e.value.status == 6 and "sdf_node_intersect" in str(e.value)
    p = parity_preset()
    p.sdf_node_intersect = 7
    sc.SetPreset(p)
    with pytest.raises(LrtError) as e:
        sc.RayQuery_NearestHitBatch(rays[:8])
    assert e.value.status == 6 and "sdf_node_intersect" in str(e.value)
    sc.SetPreset(parity_preset())
    sc.RayQuery_NearestHitBatch(rays[:8])


def test_voxel_march_limit_reports_and_recovers(cuda):
    sc, rays, want = _sbs_scene()
    sc.set_voxel_step_limit(1)
    with pytest.raises(LrtError) as e:
        sc.RayQuery_NearestHitBatch(rays)
    assert e.value.status == 5 and "voxel" in str(e.value)
    sc.set_voxel_step_limit(0)
    got = sc.RayQuery_NearestHitBatch(rays)   # same context, default limit again
    assert bit_equal(got, want).all()


def test_pipelined_host_trace_reports_limit_and_recovers(cuda):
    """Host buffers of 262,144 rays or more run through the chunked
    pipeline, whose traces share one error word: a march limit in any chunk
    is reported once, and the next call (default limit) is exact."""
    sc, rays, want = _sbs_scene()
    reps = -(-300000 // len(rays))
    big = np.ascontiguousarray(np.tile(rays, (reps, 1)))
    big_want = np.tile(want, reps)
    sc.set_voxel_step_limit(1)
    with pytest.raises(LrtError) as e:
        sc.RayQuery_NearestHitBatch(big)
    assert e.value.status == 5 and "voxel" in str(e.value)
    sc.set_voxel_step_limit(0)
    for _ in range(2):
        got = sc.RayQuery_NearestHitBatch(big)
        assert bit_equal(got, big_want).all()


def test_recommit_and_clear(cuda):
    sc = SceneRT()
    v, t = wl.noisy_sphere(16)
    g = sc.AddGeom_Triangles3f(v, t)
    sc.AddInstance(g, wl.IDENTITY)
    sc.CommitScene()
    rays = wl.eye_rays_host(wl.camera((0, 0, 3), width=32, height=32))
    a = sc.RayQuery_NearestHitBatch(rays)
    sc.ClearScene()
    m = wl.IDENTITY.copy()
    m[12] = 5.0  # move the instance out of view
    sc.AddInstance(g, m)
    sc.CommitScene()
    b = sc.RayQuery_NearestHitBatch(rays)
    assert (a["primId"] != 0xFFFFFFFF).sum() > 100 and (b["primId"] != 0xFFFFFFFF).sum() == 0

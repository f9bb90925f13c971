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


def test_misaligned_device_pointer_is_rejected(cuda):
    torch = cuda
    sc, rays, _ = _sbs_scene()
    R = torch.zeros(len(rays) * 8 + 4, dtype=torch.float32, device="cuda")
    H = torch.zeros(len(rays) * 8, dtype=torch.float32, device="cuda")
    with pytest.raises(LrtError) as e:
        sc.trace_device(R.data_ptr() + 4, H.data_ptr(), len(rays))
    assert e.value.status == 1 and "aligned" in str(e.value)


def test_unsupported_preset_is_refused(cuda):
    sc, rays, _ = _sbs_scene()
    sc.SetPreset(default_preset())  # ANALYTIC node intersection is not on the path
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

"""lrt_trace_nearest_noalloc: the allocation-free trace for hosts that cannot
call cudaMalloc after their scene is uploaded (their GPU memory budget
belongs to their own pool, or allocation is forbidden in the frame loop).

It must give the same hits as lrt_trace_nearest — bit for bit, the tolerance
of the exact build — on two calls in a row (the shared static scratch keeps
the previous call's contents), for host and device buffers, and it must
refuse host batches larger than its static staging capacity.  This file is
collected last so that a failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from graphic_lab_task_b200 import HIT_DTYPE, SceneRT
from graphic_lab_task_b200._abi import LRT_TRACE_DEVICE_POINTERS
from graphic_lab_task_b200.lrt import lib
from helpers import bit_equal, hit_summary, load_golden

pytestmark = pytest.mark.gpu

MAX_HOST_RAYS = 16384


def _noalloc(sc, rays, hits, n, flags=0, stream=None):
    return lib().lrt_trace_nearest_noalloc(sc.h, C.c_void_p(rays), C.c_void_p(hits), n,
                                           C.c_void_p(stream) if stream else None, flags)


@pytest.mark.parametrize("name", ["sbs_small", "instanced_mix", "mesh_small"])
def test_noalloc_matches_regular_entry_point_twice(cuda, name):
    arrays, rays, want, preset = load_golden(name)
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    regular = sc.RayQuery_NearestHitBatch(rays)
    assert bit_equal(regular, want).all()
    rays = np.ascontiguousarray(rays, np.float32)
    for _ in range(2):
        got = np.zeros(len(rays), HIT_DTYPE)
        assert _noalloc(sc, rays.ctypes.data, got.ctypes.data, len(rays)) == 0, lib().lrt_last_error(sc.h)
        assert bit_equal(got, regular).all(), hit_summary(got, regular)


def test_noalloc_device_buffers_twice(cuda):
    torch = cuda
    arrays, rays, want, preset = load_golden("sbs_small")
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    regular = sc.RayQuery_NearestHitBatch(rays)
    R = torch.from_numpy(np.ascontiguousarray(rays)).cuda()
    for _ in range(2):
        H = torch.zeros(len(rays) * 8, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        st = _noalloc(sc, R.data_ptr(), H.data_ptr(), len(rays), LRT_TRACE_DEVICE_POINTERS)
        assert st == 0, lib().lrt_last_error(sc.h)
        got = H.cpu().numpy().view(HIT_DTYPE)
        assert bit_equal(got, regular).all(), hit_summary(got, regular)


def test_noalloc_refuses_batches_beyond_its_capacity(cuda):
    arrays, rays, want, preset = load_golden("hand_triangle")
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    big = np.tile(rays, (MAX_HOST_RAYS // len(rays) + 1, 1))[: MAX_HOST_RAYS + 1]
    out = np.zeros(len(big), HIT_DTYPE)
    st = _noalloc(sc, big.ctypes.data, out.ctypes.data, len(big))
    assert st == 1
    assert b"16384" in lib().lrt_last_error(sc.h)
    # exactly at capacity is accepted and matches the regular path
    ok = np.ascontiguousarray(big[:MAX_HOST_RAYS])
    got = np.zeros(len(ok), HIT_DTYPE)
    assert _noalloc(sc, ok.ctypes.data, got.ctypes.data, len(ok)) == 0
    assert bit_equal(got, sc.RayQuery_NearestHitBatch(ok)).all()

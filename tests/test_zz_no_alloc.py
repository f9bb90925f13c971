"""lrt_trace_nearest_noalloc: the allocation-free trace for hosts that cannot
call cudaMalloc after their scene is uploaded (their GPU memory budget
belongs to their own pool, or allocation is forbidden in the frame loop).

It must give the same hits as lrt_trace_nearest — bit for bit, the tolerance
of the exact build — on two calls in a row (the shared static scratch keeps
the previous call's contents), for host and device buffers; it must leave
its process's device memory unchanged from its first call on (the array is
placed at upload); it must refuse host batches larger than its static staging
capacity, work counting and a wrong current device; and a bounded-loop limit
must come back as LRT_ERR_DEVICE_LIMIT with the next calls exact again.  This
file is collected last so that a failure here never hides the other tests.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from graphic_lab_task_b200 import HIT_DTYPE, SceneRT
from graphic_lab_task_b200._abi import LRT_TRACE_COUNT_WORK, LRT_TRACE_DEVICE_POINTERS, LRT_TRACE_FAST_MATH
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


def test_noalloc_reports_the_voxel_limit_and_recovers(cuda):
    """The error word lives in the shared array and keeps the failed call's
    bits: the call that hits the limit reports LRT_ERR_DEVICE_LIMIT, and the
    next two calls (default limit) clear it and are exact."""
    arrays, rays, want, preset = load_golden("sbs_small")
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    rays = np.ascontiguousarray(rays, np.float32)
    got = np.zeros(len(rays), HIT_DTYPE)
    sc.set_voxel_step_limit(1)
    assert _noalloc(sc, rays.ctypes.data, got.ctypes.data, len(rays)) == 5
    assert b"voxel" in lib().lrt_last_error(sc.h)
    sc.set_voxel_step_limit(0)
    for _ in range(2):
        got = np.zeros(len(rays), HIT_DTYPE)
        assert _noalloc(sc, rays.ctypes.data, got.ctypes.data, len(rays)) == 0, lib().lrt_last_error(sc.h)
        assert bit_equal(got, want).all(), hit_summary(got, want)


def test_noalloc_fast_math_matches_regular_fast_math(cuda):
    arrays, rays, want, preset = load_golden("instanced_mix")
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    regular = sc.RayQuery_NearestHitBatch(rays, fast_math=True)
    rays = np.ascontiguousarray(rays, np.float32)
    for _ in range(2):
        got = np.zeros(len(rays), HIT_DTYPE)
        assert _noalloc(sc, rays.ctypes.data, got.ctypes.data, len(rays), LRT_TRACE_FAST_MATH) == 0
        assert bit_equal(got, regular).all(), hit_summary(got, regular)


def test_noalloc_refusals(cuda):
    torch = cuda
    arrays, rays, want, preset = load_golden("hand_triangle")
    sc = SceneRT(preset=preset)
    sc.upload_arrays(arrays)
    rays = np.ascontiguousarray(rays, np.float32)
    out = np.zeros(len(rays), HIT_DTYPE)
    assert _noalloc(sc, rays.ctypes.data, out.ctypes.data, len(rays), LRT_TRACE_COUNT_WORK) == 1
    assert b"COUNT_WORK" in lib().lrt_last_error(sc.h)
    if torch.cuda.device_count() > 1:
        with torch.cuda.device(1):
            assert _noalloc(sc, rays.ctypes.data, out.ctypes.data, len(rays)) == 1
        assert b"current" in lib().lrt_last_error(sc.h)
    assert _noalloc(sc, rays.ctypes.data, out.ctypes.data, len(rays)) == 0
    assert bit_equal(out, want).all()


# Run in a fresh process, so that nothing earlier in the process has traced
# or loaded a module: upload a scene, then the first allocation-free call and
# 100 more must leave this process's device memory as it was after the
# upload.  The memory is read per process from NVML (the device's free memory
# also moves when another process's context on the GPU, the test runner's
# for one, allocates), and the device's free memory must not change over the
# first call, where a module load would place memory.
_FRESH_PROCESS_CHECK = r"""
import ctypes as C, os, sys
import numpy as np, torch
import pynvml
from graphic_lab_task_b200 import HIT_DTYPE, SceneRT
from graphic_lab_task_b200.lrt import lib
from helpers import bit_equal, load_golden
pynvml.nvmlInit()


def process_memory():
    for d in range(pynvml.nvmlDeviceGetCount()):
        for p in pynvml.nvmlDeviceGetComputeRunningProcesses(pynvml.nvmlDeviceGetHandleByIndex(d)):
            if p.pid == os.getpid():
                return p.usedGpuMemory
    return None


torch.cuda.init()
arrays, rays, want, preset = load_golden("sbs_small")
sc = SceneRT(preset=preset)
sc.upload_arrays(arrays)
torch.cuda.synchronize()
rays = np.ascontiguousarray(rays, np.float32)
free0, used0 = torch.cuda.mem_get_info()[0], process_memory()
frees, used = [], []
for i in range(101):
    got = np.zeros(len(rays), HIT_DTYPE)
    st = lib().lrt_trace_nearest_noalloc(sc.h, C.c_void_p(rays.ctypes.data), C.c_void_p(got.ctypes.data),
                                         len(rays), None, 0)
    assert st == 0, lib().lrt_last_error(sc.h)
    assert bit_equal(got, want).all()
    frees.append(torch.cuda.mem_get_info()[0])
    used.append(process_memory())
print("device free after upload", free0, "after the first call", frees[0], "min/max", min(frees), max(frees),
      "; this process's memory after upload", used0, "over the calls", sorted(set(used)))
if used0 is None:  # NVML does not see this process (another pid namespace): the device's free memory
    sys.exit(0 if min(frees) == free0 == max(frees) else 3)
sys.exit(0 if frees[0] == free0 and all(u == used0 for u in used) else 3)
"""


def test_noalloc_leaves_process_device_memory_unchanged(cuda):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([root, os.path.join(root, "tests"), os.path.join(root, "oracle"),
                                         env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", _FRESH_PROCESS_CHECK], cwd=root, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr

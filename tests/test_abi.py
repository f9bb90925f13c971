"""The C-ABI library loads, exports every declared symbol and reports errors
by status code and message (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from graphic_lab_task_b200 import LrtError, SceneRT, default_preset, lib
from graphic_lab_task_b200._abi import HIT_DTYPE, Preset
from graphic_lab_task_b200.lrt import EXPORTED

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = set()
    for h in os.listdir(INCLUDE):
        src = open(os.path.join(INCLUDE, h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+char\s*\*|lrt_status|double)\s+(lrt_\w+)\s*\(", src, flags=re.M))
    return names


def test_every_declared_symbol_is_exported():
    L = lib()
    declared = declared_functions()
    assert len(declared) >= 25
    missing = [n for n in sorted(declared) if not hasattr(L, n)]
    assert not missing, missing
    assert set(EXPORTED) <= declared, set(EXPORTED) - declared


def test_library_is_the_in_tree_cuda_build():
    L = lib()
    path = os.path.realpath(L._name)
    assert path.endswith(os.path.join("graphic_lab_task_b200", "liblrt_b200.so"))
    # the library carries sm_100a device code
    blob = open(path, "rb").read()
    assert b"sm_100a" in blob


def test_default_preset_matches_reference():
    p = Preset()
    assert lib().lrt_default_preset(C.byref(p)) == 0
    d = default_preset()
    for f, _ in Preset._fields_:
        assert getattr(p, f) == pytest.approx(getattr(d, f)), f
    # getDefaultPreset: ANALYTIC node intersection, VERTEX normals
    assert p.sdf_node_intersect == 1 and p.normal_mode == 1 and p.render_mode == 1


def test_errors_are_status_codes_with_messages():
    sc = SceneRT()
    with pytest.raises(LrtError) as e:
        sc.RayQuery_NearestHitBatch(np.zeros((4, 8), np.float32))
    assert e.value.status == 3 and "CommitScene" in str(e.value)
    with pytest.raises(LrtError) as e:
        sc.AddInstance(5, np.eye(4, dtype=np.float32).reshape(16))
    assert e.value.status == 1 and "geometry 5" in str(e.value)
    with pytest.raises(LrtError) as e:
        sc.AddGeom_Triangles3f(np.zeros((3, 3), np.float32), np.array([0, 1, 7], np.uint32))
    assert "index 7" in str(e.value)
    with pytest.raises(LrtError):
        sc.CommitScene(host_only=True)  # no instances
    assert lib().lrt_scene_destroy(None) == 0
    assert lib().lrt_trace_nearest(None, None, None, 0, None, 0) == 1


def test_single_ray_query_without_commit_fails_cleanly():
    sc = SceneRT()
    with pytest.raises(LrtError):
        sc.RayQuery_NearestHit(np.zeros(4, np.float32), np.array([0, 0, 1, 1e9], np.float32))
    with pytest.raises(LrtError):
        sc.RayQuery_AnyHit(np.zeros(4, np.float32), np.array([0, 0, 1, 1e9], np.float32))


def test_hit_layout():
    h = np.zeros(1, HIT_DTYPE)
    assert h.itemsize == 32
    assert HIT_DTYPE.fields["coords"][1] == 16


def test_pipeline_chunk_schedule_mirror():
    """graphic_lab_task_b200.lrt.pipeline_chunks mirrors the library's chunk
    schedule of host-buffer traces: sizes sum to n, ramp up and down."""
    from graphic_lab_task_b200.lrt import PIPE_CHUNK, PIPE_CHUNK_MIN, pipeline_chunks
    for n in (1, 1000, 262144, 300001, 1000003, 2073600, 16777216):
        c = pipeline_chunks(n)
        assert sum(c) == n and all(0 < x <= PIPE_CHUNK for x in c)
    c = pipeline_chunks(2073600)
    assert c[0] == PIPE_CHUNK_MIN and c[-1] == PIPE_CHUNK_MIN and len(c) == 13

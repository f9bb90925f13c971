"""Multi-rank path on CPU: two gloo ranks trace replicas (with the oracle as
the stand-in compute), agree bit for bit, and reduce their times to the max
exactly as bench.py does with NCCL."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from graphic_lab_task_b200.replicas import job_throughput, max_over_ranks, shard_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, out_dir):
    import sys
    import time
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import pyoracle as po
    from graphic_lab_task_b200 import workloads as wl
    from graphic_lab_task_b200 import SceneRT
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = SceneRT()
        v, t = wl.noisy_sphere(24, seed=4)
        sc.AddInstance(sc.AddGeom_Triangles3f(v, t), wl.IDENTITY)
        sc.CommitScene(host_only=True)
        rays = wl.eye_rays_host(wl.camera((0, 0, 3), width=32, height=32))
        dist.barrier()
        t0 = time.perf_counter()
        hits = po.port_trace(sc.export_arrays(), rays, threads=1)
        ms = (time.perf_counter() - t0) * 1e3 + 10.0 * rank  # rank 1 is slower by 10 ms
        (mx,) = max_over_ranks([ms])
        b, e = shard_range(len(rays), rank, world)
        np.savez(os.path.join(out_dir, "r%d.npz" % rank), hits=hits.view(np.uint8), ms=ms, mx=mx, b=b, e=e)
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    r0 = np.load(tmp_path / "r0.npz")
    r1 = np.load(tmp_path / "r1.npz")
    assert np.array_equal(r0["hits"], r1["hits"])          # replicas agree
    assert float(r0["mx"]) == float(r1["mx"]) == max(float(r0["ms"]), float(r1["ms"]))
    assert (int(r0["b"]), int(r0["e"]), int(r1["b"]), int(r1["e"])) == (0, 512, 512, 1024)
    v = job_throughput(1024, world, 1, float(r0["mx"]))
    assert abs(v - 2 * 1024 / (float(r0["mx"]) * 1e-3) / 1e6) < 1e-9

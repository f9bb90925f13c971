"""Multi-GPU form of the ray query: independent replicas.

Rays are independent and the reference has no exchange step, so N ranks each
hold the whole scene and trace their own batch; there is no collective on the
data path.  The only cross-rank operations are a barrier before timing and a
max-reduction of the measured times (the job takes as long as its slowest
rank).  These helpers are shared by bench.py (NCCL, CUDA tensors) and the
world-size-2 gloo tests (CPU tensors).
"""
import torch
import torch.distributed as dist


def max_over_ranks(values, device=None):
    """Element-wise max of a list of floats over all ranks (identity when
    torch.distributed is not initialised)."""
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def job_throughput(rays_per_rank_per_step, world, steps, total_ms):
    """Whole-job Mrays/s: every rank traced `rays_per_rank_per_step` rays per
    step; `total_ms` is the max over ranks of the summed step times."""
    return world * rays_per_rank_per_step * steps / (total_ms * 1e-3) / 1e6


def shard_range(n, rank, world):
    """Contiguous [begin, end) share of n independent items for `rank`
    (used when a fixed ray set is split instead of replicated)."""
    per = (n + world - 1) // world
    b = min(n, rank * per)
    return b, min(n, b + per)

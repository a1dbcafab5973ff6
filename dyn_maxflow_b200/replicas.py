"""Replica runs on several GPUs of one node (one process per GPU, torchrun).

A single solve does not shard (every BFS level and push round needs a grid-wide
barrier over the whole residual graph), so multi-GPU runs are independent
replicas: each rank owns its own solver and graph copy.  The only cross-rank
step is the reduction of the per-rank timings, where the job's time is the
slowest rank's.  torch.distributed is the plumbing (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations


def reduce_max(values):
    """Element-wise max of `values` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(vals, dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.cpu().tolist()


def replica_summary(p50_ms: float, mean_ms: float, e2e_p50_ms: float, world: int) -> dict:
    """Job-level numbers of a replica run: the max over ranks of each latency, and
    the aggregate batch throughput (every rank completes one batch per step)."""
    p50, mean, e2e = reduce_max([p50_ms, mean_ms, e2e_p50_ms])
    return {"p50_ms": p50, "ms_per_step": mean, "e2e_p50_ms": e2e,
            "throughput_batches_per_s": world * 1e3 / mean if mean > 0 else 0.0}

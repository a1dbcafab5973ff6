"""The multi-GPU path is replicas only; its cross-rank step (max-over-ranks timing
and aggregate throughput) runs here as two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dyn_maxflow_b200.replicas import replica_summary, reduce_max
        # rank r reports latencies 1+r, 10+r, 2+r: the job's numbers are the slowest rank's
        out = replica_summary(1.0 + rank, 10.0 + rank, 2.0 + rank, world)
        out["raw"] = reduce_max([rank * 3.5, -rank])
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_two_rank_replica_reduction():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank in (0, 1):
        o = got[rank]
        assert o["p50_ms"] == 2.0 and o["ms_per_step"] == 11.0 and o["e2e_p50_ms"] == 3.0
        assert o["throughput_batches_per_s"] == pytest.approx(2 * 1e3 / 11.0)
        assert o["raw"] == [3.5, 0.0]


def test_single_process_is_identity():
    from dyn_maxflow_b200.replicas import reduce_max, replica_summary
    assert reduce_max([1.5, 2.5]) == [1.5, 2.5]
    assert replica_summary(1.0, 2.0, 3.0, 1)["throughput_batches_per_s"] == 500.0

"""The N > 1 path of bench.py (independent replicas, one process per GPU) on
the CPU: two gloo ranks take the maximum of their device times and report all
ranks' steps over it, as the NCCL ranks do on a GPU box."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms_local = 100.0 + 50.0 * rank   # the second replica is the slower one
        ms = bench.replica_max(ms_local, dist, "cpu")
        out[rank] = (ms, bench.replica_rate(200, ms, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0] == res[1]                       # every rank sees the same max
    ms, rate = res[0]
    assert ms == 150.0 and rate == pytest.approx(2 * 200 / 0.150)

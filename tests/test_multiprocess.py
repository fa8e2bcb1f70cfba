"""CPU: the multi-rank host logic of bench.py on 2 gloo ranks (replicas:
max-over-ranks timing, whole-job value), without a GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 * (rank + 1)          # rank 1 is the slow one
        worst = bench.max_over_ranks(local_ms, world)
        dist.barrier()
        out[rank] = (worst, bench.replica_gflops(30_000_000, 5, world, worst))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_and_value():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1]
    worst, value = out[0]
    assert worst == 20.0
    assert value == pytest.approx(2.0 * 30e6 * 5 * 2 / 0.020 / 1e9)


def test_single_rank_is_identity():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_gflops(10, 1, 1, 1e3) == pytest.approx(2e-8)

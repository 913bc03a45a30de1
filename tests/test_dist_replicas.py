"""The multi-rank path of bench.py on CPU: two gloo ranks, each timing its own
replica, reduce to the slowest rank and report the whole-job throughput."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    w, r, local = bench.setup_dist()
    assert (w, r, local) == (world, rank, rank)
    bench.barrier(w)
    per_rank_seconds = 1.0 + rank          # rank 1 is the slow one
    slowest = bench.reduce_max(per_rank_seconds, w, device="cpu")
    value = bench.aggregate_value(1000, 10, slowest, w)
    out[rank] = (slowest, value)
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_rank():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == (2.0, 2 * 1000 * 10 / 2.0)

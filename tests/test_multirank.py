"""Host logic of the multi-GPU bench on CPU ranks (gloo, world size 2).

The path shards as independent replicas (one model per GPU, no exchange
step), so the only cross-rank operations are the barrier and the max of the
per-rank device times; both are checked here without a GPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    ms = 10.0 + 5.0 * rank                    # per-rank device time
    bench.barrier(world)
    m = bench.max_over_ranks(ms, world)
    out[rank] = (m, bench.job_rate(1000, 4, m, world))
    dist.destroy_process_group()


def test_two_rank_timing_reduction():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    for r in range(world):
        m, rate = res[r]
        assert m == 15.0                       # max over ranks, same on every rank
        assert rate == pytest.approx(world * 1000 * 4 / 0.015 / 1e9)

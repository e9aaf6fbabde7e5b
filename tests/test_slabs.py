"""Host logic of the z-slab decomposition, on CPU: the cut plan, the receiver
split, the source rule, and the halo exchange between ranks (gloo, world
sizes 2 and 3, CPU tensors standing in for the device buffers that the GPU
path sends over NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT
import sgfd.slabs as sl


def test_plan_even_split_and_weights():
    assert sl.plan_cuts(110, 1) == [(0, 100)]
    assert sl.plan_cuts(110, 4) == [(0, 25), (25, 25), (50, 25), (75, 25)]
    cuts = sl.plan_cuts(110, 2, weights=[1, 3])
    assert cuts == [(0, 25), (25, 75)]
    for nz, k in [(61, 3), (394, 8), (522, 7), (25, 3)]:
        cuts = sl.plan_cuts(nz, k)
        assert cuts[0][0] == 0 and sum(n for _, n in cuts) == nz - 10
        assert all(z1 == z0 + n for (z0, n), (z1, _) in zip(cuts, cuts[1:]))
        assert all(n >= sl.MIN_PLANES for _, n in cuts)
    with pytest.raises(ValueError):
        sl.plan_cuts(24, 3)                       # 14 computed planes: no room for 3 slabs of 5


def test_plan_moves_cuts_away_from_the_source():
    nz = 110                                      # 100 computed planes, even cut at 50
    for src_z in range(5, 105):
        cuts = sl.plan_cuts(nz, 2, src_z=src_z)
        sl.check_source(cuts, src_z)              # raises if the source is within 5 planes of a cut
        assert abs(cuts[1][0] - 50) <= 11
    cuts = sl.plan_cuts(nz, 2, src_z=5 + 50)
    assert cuts == [(0, 45), (45, 55)]            # the nearer of the two admissible cuts
    with pytest.raises(ValueError):
        sl.check_source([(0, 50), (50, 50)], 5 + 47)
    with pytest.raises(ValueError):
        sl.plan_cuts(26, 3, src_z=5 + 8)          # 16 planes, no admissible cut near the source


def test_receiver_split_and_source_slab():
    cuts = [(0, 12), (12, 14), (26, 9)]
    xyz = np.array([[7, 8, 5], [7, 8, 16], [7, 8, 17], [9, 9, 30], [9, 9, 31], [6, 6, 39]], np.int32)
    comp = np.arange(6, dtype=np.int32)
    parts = sl.split_receivers(cuts, xyz, comp)
    assert [list(p[0]) for p in parts] == [[0, 1], [2, 3], [4, 5]]
    assert [list(p[1][:, 2]) for p in parts] == [[5, 16], [5, 18], [5, 13]]
    assert list(parts[1][2]) == [2, 3]
    assert [sl.source_slab(cuts, z) for z in (5, 16, 17, 30, 31, 39)] == [0, 0, 1, 1, 2, 2]
    with pytest.raises(ValueError):
        sl.source_slab(cuts, 40)                  # the top frame


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "staggered-grid_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    import sgfd.slabs as slabs
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n = 7
    send_lo = torch.full((n,), 100.0 * rank + 1.0)   # this rank's planes next to its lower cut
    send_hi = torch.full((n,), 100.0 * rank + 2.0)
    recv_lo = torch.full((n,), -1.0)
    recv_hi = torch.full((n,), -1.0)
    for _ in range(2):                                # the two exchanges of a step, same pairing
        slabs.exchange_remote(send_lo, send_hi, recv_lo, recv_hi, rank, world)
    out[rank] = (recv_lo.tolist(), recv_hi.tolist())
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_between_ranks(world):
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
        lo, hi = res[r]
        # the frame below a slab holds the lower neighbour's planes next to the cut (its "high" side)
        assert lo == ([100.0 * (r - 1) + 2.0] * 7 if r > 0 else [-1.0] * 7)
        assert hi == ([100.0 * (r + 1) + 1.0] * 7 if r < world - 1 else [-1.0] * 7)

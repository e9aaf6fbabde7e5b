"""z-slabs on one GPU: the model cut along z into 2 or 3 handles that trade
5-plane halos between the half steps gives the whole model's traces and
final wavefields BIT FOR BIT (the whole-model run is itself pinned bit for bit
to the oracle by test_gpu_parity.py).  Cases cover a cut moved away from the
source, a slab lying entirely inside the bottom z-PML band, slabs crossing the
band edges, several z chunks per slab, both kernel families and both rounding
modes."""
import numpy as np
import pytest

from helpers import make_solver
import sgfd
import sgfd.slabs as sl
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu

CASES = [
    # (id, small_random_case arguments, slabs or explicit cuts, kernel, z chunk, arith, source override)
    ("two_zmarch_ref", dict(), 2, sgfd.KERNEL_ZMARCH, 0, sgfd.ARITH_REF, None),
    ("three_simple_fast", dict(quirks=sgfd.QUIRKS_FIXED, damping=sgfd.DAMP_LOGR), 3, sgfd.KERNEL_SIMPLE, 0,
     sgfd.ARITH_FAST, None),
    ("pml_slab_zmarch_chunk7", dict(nx=40, ny=34, nz=60, pml=6, nt=50), [(0, 5), (5, 20), (25, 25)],
     sgfd.KERNEL_ZMARCH, 7, sgfd.ARITH_REF, (21, 18, 45)),
    ("three_zmarch_fast_logr", dict(nx=45, ny=38, nz=70, pml=8, nt=40, damping=sgfd.DAMP_LOGR,
                                    quirks=sgfd.QUIRKS_FIXED), 3, sgfd.KERNEL_ZMARCH, 0, sgfd.ARITH_FAST, None),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_slabs_equal_whole_model(case):
    _, kw, slabs, kernel, zchunk, arith, src = case
    w = wl.small_random_case(**kw)
    w.cfg["arith"] = arith
    if src is not None:
        w.src = src
    cuts = sl.plan_cuts(w.cfg["nz"], slabs, src_z=w.src[2]) if isinstance(slabs, int) else slabs
    with make_solver(w, kernel=kernel) as s:
        if zchunk:
            s.set_zchunk(zchunk)
        s.run(0, w.nt)
        s.synchronize()
        want_tr = s.traces()
        want = [s.field(f) for f in range(9)]
    cfg = sgfd.default_config(**{**w.cfg, "kernel": kernel})
    with sl.SlabModel(cfg, cuts) as m:
        assert [sb.kernel_name() for sb in m.slabs] == [("zmarch" if kernel == sgfd.KERNEL_ZMARCH else "simple")] * len(cuts)
        if zchunk:
            for sb in m.slabs:
                sb.set_zchunk(zchunk)
        m.set_medium(w.b, w.lam, w.mu)
        m.set_source(*w.src)
        m.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
        m.run(0, w.nt, w.wavelet)
        m.synchronize()
        tr = m.traces()
        assert np.abs(want_tr).max() > 0
        np.testing.assert_array_equal(tr, want_tr)
        for f in range(9):
            np.testing.assert_array_equal(m.field(f), want[f], err_msg=sgfd.FIELD_NAMES[f])


def test_slab_cell_counts_add_up():
    """The slabs' PML cells (counted in the whole model's bands) add up to the whole model's."""
    w = wl.small_random_case(nx=40, ny=34, nz=60, pml=6, nt=4)
    cuts = [(0, 5), (5, 20), (25, 25)]
    cfg = sgfd.default_config(**w.cfg)
    with make_solver(w) as s:
        n_int, n_pml = s.cell_counts()
    with sl.SlabModel(cfg, cuts) as m:
        counts = [sb.cell_counts() for sb in m.slabs]
    assert sum(c[0] for c in counts) == n_int
    assert sum(c[1] for c in counts) == n_pml
    assert counts[0][0] == 0                      # the first slab lies inside the bottom z band


def test_slab_configuration_errors():
    w = wl.small_random_case(nt=4)
    cfg = sgfd.default_config(**w.cfg)
    bad = [dict(nz_total=cfg.nz, z_offset=0, nz=14),                   # 4 computed planes: too thin
           dict(nz_total=cfg.nz, z_offset=cfg.nz - 10 - 4, nz=15),     # runs past the model's top
           dict(nz_total=0, z_offset=3),                               # offset without a whole model
           dict(nz_total=cfg.nz, z_offset=0, nz=20, storage=sgfd.STORE_F16)]
    for kw in bad:
        c = sgfd.default_config(**{**w.cfg, **kw})
        with pytest.raises(sgfd.SgfdError):
            sgfd.Solver(c)
    c = sl.slab_config(cfg, 0, 20)
    with sgfd.Solver(c) as s:
        px = (cfg.nx + 27 + 31) // 32 * 32                         # padded row pitch
        assert s.halo_bytes() == 3 * 5 * px * cfg.ny * 4
        with pytest.raises(sgfd.SgfdError):
            s.set_learned_strip(6, np.zeros(sgfd.lib().sgfd_mlp_param_count(), np.float32))


def _dist_worker(rank, world, port, case_kw, cuts, kernel, out):
    import os
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch
    import torch.distributed as dist
    import sgfd
    import sgfd.slabs as slabs
    import sgfd.workloads as wlm
    dist.init_process_group("gloo", rank=rank, world_size=world)
    torch.cuda.set_device(0)
    w = wlm.small_random_case(**case_kw)
    cfg = sgfd.default_config(**{**w.cfg, "kernel": kernel})
    m = slabs.DistributedSlab(cfg, cuts, rank, world, 0)
    m.set_medium(w.b, w.lam, w.mu)
    m.set_source(*w.src)
    m.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
    m.run(0, w.nt, w.wavelet)
    m.synchronize()
    out[rank] = (m.rec_parts[rank][0], m.traces(), [m.own_planes(f) for f in range(9)])
    m.close()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,kernel", [(2, sgfd.KERNEL_ZMARCH), (3, sgfd.KERNEL_SIMPLE)],
                         ids=["two_ranks_zmarch", "three_ranks_simple"])
def test_distributed_slabs_on_one_gpu(world, kernel):
    """The one-slab-per-rank form end to end: world_size ranks (processes)
    share this GPU, each holding one slab, and trade halos through host memory
    over gloo (no kernel waits on another process).  Its step sequence, the
    send/recv pairing and the pack/unpack sides are those of the NCCL form;
    the stitched traces and fields equal the whole model's bit for bit."""
    import socket
    import torch.multiprocessing as mp
    kw = dict(nx=41, ny=37, nz=56, pml=5, nt=40)
    w = wl.small_random_case(**kw)
    cuts = sl.plan_cuts(w.cfg["nz"], world, src_z=w.src[2])
    with make_solver(w, kernel=kernel) as s:
        s.run(0, w.nt)
        s.synchronize()
        want_tr = s.traces()
        want = [s.field(f) for f in range(9)]
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_dist_worker, args=(r, world, port, kw, cuts, kernel, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(out)
    covered = 0
    for r in range(world):
        idx, tr, planes = res[r]
        np.testing.assert_array_equal(tr, want_tr[idx])
        covered += len(idx)
        for f, (z0, a) in enumerate(planes):
            np.testing.assert_array_equal(a, want[f][5 + z0:5 + z0 + a.shape[0]], err_msg=sgfd.FIELD_NAMES[f])
    assert covered == len(w.rec_comp) and np.abs(want_tr).max() > 0


@pytest.mark.parametrize("kernel,zchunk", [(sgfd.KERNEL_ZMARCH, 0), (sgfd.KERNEL_ZMARCH, 7), (sgfd.KERNEL_ZMARCH, 3),
                                           (sgfd.KERNEL_SIMPLE, 0)], ids=["zmarch", "zmarch_chunk7", "zmarch_chunk3",
                                                                          "simple"])
def test_half_step_parts_equal_steps(kernel, zchunk):
    """A whole model stepped as velocity inner, velocity outer, stress inner,
    stress outer (the slabs' overlapped order) equals sgfd_run bit for bit."""
    w = wl.small_random_case(nx=39, ny=35, nz=44, pml=5, nt=30)
    outs = []
    for split in (False, True):
        with make_solver(w, kernel=kernel) as s:
            if zchunk:
                s.set_zchunk(zchunk)
            if split:
                for it in range(w.nt):
                    for phase in (sgfd.PHASE_VELOCITY, sgfd.PHASE_STRESS):
                        s.step_phase(it, float(w.wavelet[it]), phase, sgfd.PART_INNER)
                        s.step_phase(it, float(w.wavelet[it]), phase, sgfd.PART_OUTER)
            else:
                s.run(0, w.nt)
            s.synchronize()
            outs.append((s.traces(), [s.field(f) for f in range(9)]))
    np.testing.assert_array_equal(outs[1][0], outs[0][0])
    for f in range(9):
        np.testing.assert_array_equal(outs[1][1][f], outs[0][1][f], err_msg=sgfd.FIELD_NAMES[f])
    assert np.abs(outs[0][0]).max() > 0


def test_slab_checkpoints_resume_and_keep_their_place():
    """Each slab checkpoints on its own; a fresh set of slabs resumed from them
    ends bit-identical to the uninterrupted run, and a slab's checkpoint does
    not load into another slab (its place in the whole model is recorded)."""
    w = wl.small_random_case(nx=38, ny=34, nz=50, pml=5, nt=40)
    cfg = sgfd.default_config(**w.cfg)
    cuts = sl.plan_cuts(cfg.nz, 2, src_z=w.src[2])

    def model():
        m = sl.SlabModel(cfg, cuts)
        m.set_medium(w.b, w.lam, w.mu)
        m.set_source(*w.src)
        m.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
        return m
    with model() as m:
        m.run(0, w.nt, w.wavelet)
        m.synchronize()
        want_tr, want_vx = m.traces(), m.field(sgfd.VX)
    with model() as m:
        m.run(0, 17, w.wavelet)
        m.synchronize()
        saved = [s.checkpoint(17) for s in m.slabs]
    hd = [sgfd.checkpoint_header(b) for b in saved]
    assert [(h["nz_total"], h["z_offset"]) for h in hd] == [(cfg.nz, z0) for z0, _ in cuts]
    with model() as m:
        with pytest.raises(sgfd.SgfdError):
            m.slabs[1].restore(saved[0])
        assert [s.restore(b) for s, b in zip(m.slabs, saved)] == [17, 17]
        m.run(17, w.nt - 17, w.wavelet)
        m.synchronize()
        np.testing.assert_array_equal(m.traces(), want_tr)
        np.testing.assert_array_equal(m.field(sgfd.VX), want_vx)

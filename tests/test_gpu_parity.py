"""GPU vs CPU oracle on the same seeded inputs, through the C ABI.

FP32 contract: the kernels and the oracle perform the same rounded operations
(explicit FMAs, IEEE division and square root, no flush-to-zero), so traces and
final wavefields must agree BIT FOR BIT.  The FP64 oracle gives each case's
error against exact arithmetic (reported, bounded at 1e-4 relative L2)."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import make_solver, run_oracle
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu

CASES = [
    dict(quirks=sgfd.QUIRKS_REF, damping=sgfd.DAMP_REFGPU),
    dict(quirks=sgfd.QUIRKS_FIXED, damping=sgfd.DAMP_LOGR),
    dict(quirks=sgfd.QUIRKS_FIXED, damping=sgfd.DAMP_REFCPU, nx=31, ny=29, nz=27, pml=3),
    dict(quirks=sgfd.QUIRKS_REF, damping=sgfd.DAMP_LOGR, nx=23, ny=22, nz=21, pml=1, nt=40),
    dict(quirks=sgfd.QUIRKS_REF, damping=sgfd.DAMP_REFGPU, nx=70, ny=36, nz=33, pml=8, nt=50),
    # full 32x16 tiles with interior-only tile-planes, several z chunks
    dict(quirks=sgfd.QUIRKS_FIXED, damping=sgfd.DAMP_LOGR, nx=90, ny=60, nz=50, pml=6, nt=45, nrec=60),
    # a tall interior core: most tile-planes take the interior-only path
    dict(quirks=sgfd.QUIRKS_REF, damping=sgfd.DAMP_REFGPU, nx=100, ny=58, nz=64, pml=4, nt=30, nrec=6),
]
# (id, kernel family, tile rows, z chunk, tile columns)
KERNELS = [("simple", sgfd.KERNEL_SIMPLE, 0, 0, 32), ("zmarch", sgfd.KERNEL_ZMARCH, 8, 0, 32),
           ("zmarch_chunk7", sgfd.KERNEL_ZMARCH, 8, 7, 32), ("zmarch_rows16", sgfd.KERNEL_ZMARCH, 16, 0, 32),
           ("zmarch_rows16_chunk5", sgfd.KERNEL_ZMARCH, 16, 5, 32),
           ("zmarch_pairs", sgfd.KERNEL_ZMARCH, 8, 0, 64), ("zmarch_pairs_chunk6", sgfd.KERNEL_ZMARCH, 8, 6, 64)]


def _ids(c):
    return "_".join(f"{k}{v}" for k, v in c.items())


@pytest.mark.parametrize("arith", [sgfd.ARITH_REF, sgfd.ARITH_FAST], ids=["ref", "fast"])
@pytest.mark.parametrize("kernel", KERNELS, ids=[k[0] for k in KERNELS])
@pytest.mark.parametrize("case", CASES, ids=[_ids(c) for c in CASES])
def test_bit_exact_vs_oracle(case, kernel, arith):
    w = wl.small_random_case(**case)
    w.cfg["arith"] = arith
    o = run_oracle(w)
    with make_solver(w, kernel=kernel[1]) as s:
        assert s.kernel_name() == kernel[0].split("_")[0]
        if kernel[2]:
            s.set_tile(kernel[4], kernel[2], kernel[3])
            assert s.tile()[:2] == (kernel[4], kernel[2])
        s.run(0, w.nt)
        s.synchronize()
        tr = s.traces()
        np.testing.assert_array_equal(tr, o.traces().astype(np.float32))
        for fid in range(9):
            g = s.field(fid)
            np.testing.assert_array_equal(g, o.field(fid).astype(np.float32), err_msg=sgfd.FIELD_NAMES[fid])
    # error of the FP32 path against FP64 arithmetic
    o64 = run_oracle(w, fp64=True)
    err = rel_l2(tr, o64.traces())
    assert err < 1e-4, err


def test_default_kernel_is_zmarch():
    w = wl.small_random_case(nt=2)
    with make_solver(w) as s:
        assert s.kernel_name() == "zmarch"
        assert s.launches_per_step() == 2


def test_step_api_equals_run_api():
    w = wl.small_random_case(nt=30)
    with make_solver(w) as a, make_solver(w) as b:
        a.run(0, w.nt)
        for it in range(w.nt):
            b.step(it, float(w.wavelet[it]))
        a.synchronize(); b.synchronize()
        np.testing.assert_array_equal(a.traces(), b.traces())
        np.testing.assert_array_equal(a.field(sgfd.TXX), b.field(sgfd.TXX))


@pytest.mark.parametrize("kern,cols", [(sgfd.KERNEL_SIMPLE, 0), (sgfd.KERNEL_ZMARCH, 32), (sgfd.KERNEL_ZMARCH, 64)],
                         ids=["simple", "zmarch", "zmarch_pairs"])
def test_graph_replay_equals_direct_launches(kern, cols):
    """sgfd_run with CUDA graphs (16-step replays driven by a device step
    counter, remainder launched directly) against direct launches: bit-equal
    traces and fields, for one long run, for runs split at arbitrary steps, and
    after a receiver change that forces a new capture."""
    w = wl.small_random_case(nt=77, nrec=24)
    with make_solver(w, kernel=kern) as a, make_solver(w, kernel=kern) as b, make_solver(w, kernel=kern) as c:
        if cols:
            for s in (a, b, c):
                s.set_tile(cols, 8)
        a.run(0, w.nt, graph=False)
        b.prepare_run()
        b.run(0, w.nt, graph=True)
        for it0, n in ((0, 17), (17, 3), (20, 32), (52, 25)):
            c.run(it0, n, graph=True)
        for s in (a, b, c):
            s.synchronize()
        np.testing.assert_array_equal(b.traces(), a.traces())
        np.testing.assert_array_equal(c.traces(), a.traces())
        for fid in range(9):
            np.testing.assert_array_equal(b.field(fid), a.field(fid))
            np.testing.assert_array_equal(c.field(fid), a.field(fid))
        assert b.run_launches(w.nt, True) == w.nt * b.launches_per_step() + 1 + w.nt // 16
        assert b.run_launches(w.nt, False) == w.nt * b.launches_per_step()
        # new receivers: the captured graph no longer matches and is re-captured
        xyz = w.rec_xyz[::-1].copy()
        for s in (a, b):
            s.reset()
            s.set_receivers(xyz, w.rec_comp, w.nt)
        a.run(0, w.nt, graph=False)
        b.run(0, w.nt, graph=True)
        np.testing.assert_array_equal(b.traces(), a.traces())


def test_source_inside_pml_matches_oracle():
    """A source in the PML is overwritten by the split sum at the next stress
    update, as in the reference (splits are the state there)."""
    w = wl.small_random_case(nt=25)
    w.src = (6, 7, 8)
    o = run_oracle(w)
    for kern, cols in ((sgfd.KERNEL_SIMPLE, 0), (sgfd.KERNEL_ZMARCH, 32), (sgfd.KERNEL_ZMARCH, 64)):
        with make_solver(w, kernel=kern) as s:
            if cols:
                s.set_tile(cols, 8)
            s.run(0, w.nt)
            np.testing.assert_array_equal(s.traces(), o.traces().astype(np.float32))
            np.testing.assert_array_equal(s.field(sgfd.TXX), o.field(sgfd.TXX).astype(np.float32))


def test_fast_arithmetic_within_tolerance_of_reference_rounding():
    """FAST (coefficients pre-divided by the cell size) against the reference's
    rounding (REF) on the same inputs: relative L2 of traces and final fields
    below 1e-5, the north-star parity tolerance."""
    w = wl.small_random_case(nx=60, ny=56, nz=52, pml=8, nt=200, nrec=40)
    o = run_oracle(w)          # REF rounding
    w.cfg["arith"] = sgfd.ARITH_FAST
    with make_solver(w) as s:
        s.run(0, w.nt)
        assert rel_l2(s.traces(), o.traces()) < 1e-5
        for fid in (sgfd.VX, sgfd.TXX, sgfd.TYZ):
            assert rel_l2(s.field(fid), o.field(fid)) < 1e-5


@pytest.mark.parametrize("arith", [sgfd.ARITH_REF, sgfd.ARITH_FAST], ids=["ref", "fast"])
@pytest.mark.parametrize("kernel", KERNELS, ids=[k[0] for k in KERNELS])
def test_extreme_magnitudes_bit_exact(kernel, arith):
    """Initial wavefields whose magnitudes span 1e-45 .. 2e31 (subnormals,
    zeros of both signs, values whose difference sums exceed 2^100): the
    divisions of the reference's rounding take their fallback paths in some
    warps and the fast ones in others, and every kernel stays bit-exact with
    the oracle's IEEE divisions."""
    w = wl.small_random_case(nx=70, ny=40, nz=36, pml=5, nt=3, nrec=30)
    w.cfg["arith"] = arith
    w.src = (-1, -1, -1)
    rng = np.random.default_rng(31)
    fields = []
    for _ in range(9):
        e = rng.uniform(-45.0, 31.3, w.shape)
        f = (10.0 ** e) * rng.choice([-1.0, 1.0], w.shape)
        f[rng.random(w.shape) < 0.1] = 0.0
        f[rng.random(w.shape) < 0.02] = -0.0
        f[:5], f[-5:], f[:, :5], f[:, -5:], f[:, :, :5], f[:, :, -5:] = 0, 0, 0, 0, 0, 0   # the zero frame
        fields.append(f.astype(np.float32))
    import oracle_py
    o = oracle_py.Oracle(w.cfg)
    o.set_medium(w.b, w.lam, w.mu)
    o.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
    for k in range(9):
        o.set_field(k, fields[k])
    o.run(np.zeros(w.nt), 0, w.nt)
    cfg = sgfd.default_config(**{**w.cfg, "kernel": kernel[1]})
    with sgfd.Solver(cfg) as s:
        s.set_medium(w.b, w.lam, w.mu)
        s.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
        if kernel[2]:
            s.set_tile(kernel[4], kernel[2], kernel[3])
        for k in range(9):
            s.set_field(k, fields[k])
        for it in range(w.nt):
            s.step(it, 0.0)
        s.synchronize()
        np.testing.assert_array_equal(s.traces(), o.traces().astype(np.float32))
        for fid in range(9):
            np.testing.assert_array_equal(s.field(fid), o.field(fid).astype(np.float32),
                                          err_msg=sgfd.FIELD_NAMES[fid])
    o.close()

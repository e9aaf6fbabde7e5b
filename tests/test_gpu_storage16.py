"""16-bit wavefield storage (BF16 and FP16 with per-field power-of-two
scales) against the oracle's emulation of the same storage: bit-exact traces
and fields, including across the scale changes; graph replay and checkpoints
keep it bit-exact; error against FP64 reported and bounded."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import make_solver, run_oracle
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu

STORES = [(sgfd.STORE_BF16, "bf16"), (sgfd.STORE_F16, "f16")]


def _case(storage, **kw):
    w = wl.small_random_case(**kw)
    w.cfg["storage"] = storage
    return w


# (name, kernel family, tile columns (0: the default 32 x 8), z chunk)
FAMILIES = [("zmarch", sgfd.KERNEL_AUTO, 0, 0), ("zmarch_chunk6", sgfd.KERNEL_AUTO, 32, 6),
            ("zmarch_pairs", sgfd.KERNEL_AUTO, 64, 0), ("zmarch_pairs_chunk6", sgfd.KERNEL_AUTO, 64, 6),
            ("simple", sgfd.KERNEL_SIMPLE, 0, 0)]


@pytest.mark.parametrize("family", FAMILIES, ids=[f[0] for f in FAMILIES])
@pytest.mark.parametrize("arith", [sgfd.ARITH_REF, sgfd.ARITH_FAST], ids=["ref", "fast"])
@pytest.mark.parametrize("store", STORES, ids=[s[1] for s in STORES])
def test_bit_exact_vs_oracle_emulation(store, arith, family):
    """The z-marching kernels (32 x 8 tiles: 16-bit boxes staged by TMA and
    widened once per plane; 64 x 8 tiles: read back per tap) and the per-cell
    kernels all equal the oracle's emulation bit for bit."""
    w = _case(store[0], nt=110, nrec=36)    # scales re-chosen after steps 0, 1, 3, 7, 15, 31, 49, 99
    w.cfg["arith"] = arith
    o = run_oracle(w)
    with make_solver(w, kernel=family[1]) as s:
        assert s.kernel_name() == family[0].split("_")[0]
        if family[2]:
            s.set_tile(family[2], 8, family[3])
        assert s.tile()[0] in ((family[2] or 32),) or family[1] == sgfd.KERNEL_SIMPLE
        s.run(0, w.nt)
        s.synchronize()
        np.testing.assert_array_equal(s.traces(), o.traces().astype(np.float32))
        for fid in range(9):
            np.testing.assert_array_equal(s.field(fid), o.field(fid).astype(np.float32),
                                          err_msg=sgfd.FIELD_NAMES[fid])


@pytest.mark.parametrize("store", STORES, ids=[s[1] for s in STORES])
def test_graph_replay_and_checkpoint_keep_16_bit_runs_exact(tmp_path, store):
    w = _case(store[0], nt=80)
    with make_solver(w) as a, make_solver(w) as b:
        a.run(0, w.nt, graph=False)
        b.run(0, 37, graph=True)
        blob = b.checkpoint(37)
        hd = sgfd.checkpoint_header(blob)
        assert hd["storage"] == store[0] and any(hd["scale_exponents"])
        with make_solver(w) as c:
            assert c.restore(blob) == 37
            c.run(37, w.nt - 37, graph=True)
            np.testing.assert_array_equal(c.traces(), a.traces())
            for fid in range(9):
                np.testing.assert_array_equal(c.field(fid), a.field(fid))
        b.run(37, w.nt - 37, graph=True)
        np.testing.assert_array_equal(b.traces(), a.traces())


def test_16_bit_error_against_fp64():
    """Relative L2 of all traces against FP64 arithmetic after 300 steps."""
    base = wl.small_random_case(nt=300, nrec=48)
    o64 = run_oracle(base, fp64=True)
    with make_solver(base) as s32:
        s32.run(0, base.nt)
        e32 = rel_l2(s32.traces(), o64.traces())
    errs = {}
    for st, name in STORES:
        w = _case(st, nt=300, nrec=48)
        with make_solver(w) as s:
            s.run(0, w.nt)
            errs[name] = rel_l2(s.traces(), o64.traces())
    print(f"rel-L2 vs FP64: fp32 {e32:.2e}, bf16 {errs['bf16']:.2e}, f16 {errs['f16']:.2e}")
    assert e32 < 1e-5
    assert errs["f16"] < 1e-2 and errs["bf16"] < 5e-2
    assert errs["f16"] < errs["bf16"]


@pytest.mark.parametrize("cols", [32, 64], ids=["32x8", "64x8"])
@pytest.mark.parametrize("store", STORES, ids=[s[1] for s in STORES])
def test_16_bit_zmarch_large_interior_matches_oracle(store, cols):
    """A case with interior-only tile-planes and several z chunks: the
    interior paths of both 16-bit tilings equal the oracle's emulation too."""
    w = wl.small_random_case(nx=150, ny=60, nz=70, pml=4, nt=60, nrec=30)
    w.cfg["storage"] = store[0]
    o = run_oracle(w)
    with make_solver(w) as s:
        assert s.kernel_name() == "zmarch" and s.tile()[:2] == (32, 8)
        s.set_tile(cols, 8, 0)
        assert s.tile()[:2] == (cols, 8)
        s.run(0, w.nt)
        np.testing.assert_array_equal(s.traces(), o.traces().astype(np.float32))
        for fid in (sgfd.VX, sgfd.TXX, sgfd.TYZ):
            np.testing.assert_array_equal(s.field(fid), o.field(fid).astype(np.float32))


def test_16_bit_handles_reject_what_needs_fp32():
    w = _case(sgfd.STORE_F16, nt=20)
    with make_solver(w, kernel=sgfd.KERNEL_ZMARCH) as z:
        assert z.kernel_name() == "zmarch"
        with pytest.raises(sgfd.SgfdError) as e:
            z.set_tile(32, 16)                      # 16-bit boxes on 32 x 8 and 64 x 8 tiles only
        assert e.value.code == sgfd.ERR_UNSUPPORTED
    with make_solver(w, kernel=sgfd.KERNEL_SIMPLE) as s:
        with pytest.raises(sgfd.SgfdError) as e:
            s.set_audit(5, 0, 4)
        assert e.value.code == sgfd.ERR_UNSUPPORTED
        with pytest.raises(sgfd.SgfdError):
            s.set_kernel(sgfd.KERNEL_ZMARCH)        # created on the per-cell family
        s.run(0, 20)
        k, st = s.energy()
        k2, st2 = s.energy_noalloc()
        assert k > 0 and st > 0 and (k, st) == (k2, st2)
        assert s.launches_per_step() == 2 + 1 + 2 + 3

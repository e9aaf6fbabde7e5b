"""Batches of uneven models (sgfd_batch_*) and the launch-shape autotuner,
through the C ABI: every model of a batch ends bit for bit where the same
model run alone ends."""
import numpy as np
import pytest

from helpers import make_solver
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu


def _models():
    return [wl.small_random_case(nx=37, ny=41, nz=45, pml=6, nt=45, seed=7),
            wl.small_random_case(nx=52, ny=33, nz=40, pml=4, nt=45, seed=8, quirks=sgfd.QUIRKS_FIXED,
                                 damping=sgfd.DAMP_LOGR),
            wl.small_random_case(nx=29, ny=30, nz=31, pml=3, nt=45, seed=9, damping=sgfd.DAMP_REFCPU)]


@pytest.mark.parametrize("split", [False, True], ids=["one_run", "split_runs"])
def test_batch_equals_solo_runs(split):
    ws = _models()
    solo, members = [], []
    try:
        for i, w in enumerate(ws):
            s = make_solver(w)
            s.run(0, w.nt)
            s.synchronize()
            solo.append((s.traces(), [s.field(k) for k in range(9)]))
            s.close()
            # one member on the simple family: batches mix families
            members.append(make_solver(w, kernel=sgfd.KERNEL_SIMPLE if i == 2 else sgfd.KERNEL_AUTO))
        with sgfd.Batch(members) as b:
            if split:
                for it0, n in ((0, 20), (20, 1), (21, 24)):
                    b.run(it0, n)
            else:
                b.run(0, 45)
                assert b.run_launches(45) == 45 * sum(m.launches_per_step() for m in members) + 1 + 2
            b.synchronize()
            for m, (tr, fields) in zip(members, solo):
                np.testing.assert_array_equal(m.traces(), tr)
                for k in range(9):
                    np.testing.assert_array_equal(m.field(k), fields[k], err_msg=sgfd.FIELD_NAMES[k])
    finally:
        for m in members:
            m.close()


@pytest.mark.parametrize("split", [False, True], ids=["one_run", "split_runs"])
def test_persistent_batch_equals_solo_runs(split):
    """Persistent mode: one cooperative launch per run over every model's
    (tile, z chunk) work items; every model ends bit for bit where it ends
    alone, and a run is one launch."""
    ws = _models()
    solo, members = [], []
    try:
        for w in ws:
            s = make_solver(w)
            s.run(0, w.nt)
            s.synchronize()
            solo.append((s.traces(), [s.field(k) for k in range(9)]))
            s.close()
            members.append(make_solver(w))
        with sgfd.Batch(members) as b:
            b.set_persistent(True)
            assert all(m.tile()[:2] == (32, 8) for m in members)
            if split:
                for it0, n in ((0, 20), (20, 1), (21, 24)):
                    b.run(it0, n)
            else:
                b.run(0, 45)
                assert b.run_launches(45) == 1
            b.synchronize()
            for m, (tr, fields) in zip(members, solo):
                np.testing.assert_array_equal(m.traces(), tr)
                for k in range(9):
                    np.testing.assert_array_equal(m.field(k), fields[k], err_msg=sgfd.FIELD_NAMES[k])
    finally:
        for m in members:
            m.close()


def test_persistent_batch_grid_barrier_wait_is_bounded():
    """A grid barrier that cannot complete (each barrier told to wait for more
    arrivals than there are CTAs) gives up after about a second: the launch
    ends, sgfd_batch_synchronize reports it, and the context stays usable —
    the same batch then runs correctly."""
    ws = _models()[:2]
    members = [make_solver(w) for w in ws]
    try:
        with sgfd.Batch(members) as b:
            b.set_persistent(True, barrier_ctas=1 << 20)
            b.run(0, 3)
            with pytest.raises(sgfd.SgfdError) as e:
                b.synchronize()
            assert "grid-barrier" in str(e.value)
            for m in members:
                m.reset()
            b.set_persistent(True)
            b.run(0, 10)
            b.synchronize()
            for w, m in zip(ws, members):
                with make_solver(w) as s:
                    s.run(0, 10)
                    s.synchronize()
                    np.testing.assert_array_equal(m.traces()[:, :10], s.traces()[:, :10])
                    np.testing.assert_array_equal(m.field(sgfd.TXX), s.field(sgfd.TXX))
    finally:
        for m in members:
            m.close()


def test_persistent_batch_rejects_unsupported_models():
    w = _models()[0]
    with make_solver(w, kernel=sgfd.KERNEL_SIMPLE) as s, sgfd.Batch([s]) as b:
        with pytest.raises(sgfd.SgfdError):
            b.set_persistent(True)


def test_batch_rejects_bad_input():
    w = _models()[0]
    with make_solver(w) as s:
        with pytest.raises(sgfd.SgfdError):
            sgfd.Batch([s, s])
        with pytest.raises(sgfd.SgfdError):
            sgfd.Batch([])
        with sgfd.Batch([s]) as b:
            with pytest.raises(sgfd.SgfdError) as e:
                b.run(0, w.nt + 5)          # beyond the wavelet
            assert "wavelet" in str(e.value)


def test_autotune_picks_a_candidate_and_keeps_results():
    w = wl.small_random_case(nx=70, ny=36, nz=50, pml=8, nt=40)
    with make_solver(w) as ref:
        ref.run(0, w.nt)
        ref.synchronize()
        tr = ref.traces()
    with make_solver(w) as s:
        t = s.autotune(3)
        assert t.candidates >= 2 and t.ms_per_step > 0
        assert t.kernel in (sgfd.KERNEL_SIMPLE, sgfd.KERNEL_ZMARCH) and t.tile_rows in (8, 16)
        assert s.kernel_name() == ("zmarch" if t.kernel == sgfd.KERNEL_ZMARCH else "simple")
        for k in range(9):                      # timing steps were wiped
            assert not s.field(k).any()
        s.run(0, w.nt)
        np.testing.assert_array_equal(s.traces(), tr)
        # switching families by hand is also bit-identical
        s.reset()
        s.set_kernel(sgfd.KERNEL_SIMPLE if t.kernel == sgfd.KERNEL_ZMARCH else sgfd.KERNEL_ZMARCH)
        s.run(0, w.nt)
        np.testing.assert_array_equal(s.traces(), tr)
    with make_solver(w, kernel=sgfd.KERNEL_SIMPLE) as s:
        with pytest.raises(sgfd.SgfdError) as e:
            s.set_kernel(sgfd.KERNEL_ZMARCH)
        assert e.value.code == sgfd.ERR_UNSUPPORTED
        assert s.autotune(2).kernel == sgfd.KERNEL_SIMPLE


def test_batch_mixes_storage_audit_and_families():
    """One batch holding a 16-bit model, an FP32 model with a per-step energy
    audit and an FP32 model on the per-cell kernels: each ends bit-identical
    to the same model run alone, audit history included."""
    ws = _models()
    ws[0].cfg["storage"] = sgfd.STORE_F16
    solo = []
    for i, w in enumerate(ws):
        with make_solver(w, kernel=sgfd.KERNEL_SIMPLE if i == 2 else sgfd.KERNEL_AUTO) as s:
            if i == 1:
                s.set_audit(9, sgfd.REGION_INTERIOR, 5)
            s.run(0, w.nt)
            solo.append((s.traces(), s.field(sgfd.TXX), s.audit() if i == 1 else None))
    members = []
    try:
        for i, w in enumerate(ws):
            m = make_solver(w, kernel=sgfd.KERNEL_SIMPLE if i == 2 else sgfd.KERNEL_AUTO)
            if i == 1:
                m.set_audit(9, sgfd.REGION_INTERIOR, 5)
            members.append(m)
        with sgfd.Batch(members) as b:
            b.run(0, 45)
            b.synchronize()
        for i, (m, (tr, txx, hist)) in enumerate(zip(members, solo)):
            np.testing.assert_array_equal(m.traces(), tr)
            np.testing.assert_array_equal(m.field(sgfd.TXX), txx)
            if hist is not None:
                np.testing.assert_array_equal(m.audit(), hist)
    finally:
        for m in members:
            m.close()


def test_batch_with_learned_strips():
    """Two models with a learned absorbing strip (pml = 0, the network on the
    tensor cores) and one with a split-field PML in one batch: each ends bit
    for bit where the same model run alone ends."""
    rng = np.random.default_rng(12)
    p = (rng.standard_normal(sgfd.MLP_PARAMS) * 0.05).astype(np.float32)
    ws = [wl.small_random_case(nx=40, ny=44, nz=38, pml=0, nt=45, seed=11),
          wl.small_random_case(nx=36, ny=39, nz=42, pml=0, nt=45, seed=12),
          wl.small_random_case(nx=37, ny=41, nz=45, pml=6, nt=45, seed=7)]

    def build(w):
        s = make_solver(w)
        if w.cfg["pml"] == 0:
            s.set_learned_strip(6, p)
        return s

    solo, members = [], []
    try:
        for w in ws:
            with build(w) as s:
                s.run(0, w.nt)
                solo.append((s.traces(), [s.field(k) for k in range(9)]))
        members = [build(w) for w in ws]
        assert members[0].launches_per_step() == members[2].launches_per_step() + 2
        with sgfd.Batch(members) as b:
            b.run(0, 45)
            b.synchronize()
        for m, (tr, fields) in zip(members, solo):
            np.testing.assert_array_equal(m.traces(), tr)
            for k in range(9):
                np.testing.assert_array_equal(m.field(k), fields[k], err_msg=sgfd.FIELD_NAMES[k])
    finally:
        for m in members:
            m.close()

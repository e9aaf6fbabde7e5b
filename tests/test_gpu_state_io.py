"""Checkpoint / resume and the multi-component station files, through the C ABI.

A run stopped at step k, checkpointed, and resumed on a fresh handle must end
bit for bit where the uninterrupted run ends (traces and all 9 fields)."""
import os

import numpy as np
import pytest

from helpers import make_solver
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kern", [sgfd.KERNEL_SIMPLE, sgfd.KERNEL_ZMARCH], ids=["simple", "zmarch"])
@pytest.mark.parametrize("via", ["file", "bytes"])
def test_resume_from_checkpoint_is_bit_exact(tmp_path, kern, via):
    w = wl.small_random_case(nt=70, nrec=30)
    k = 33
    with make_solver(w, kernel=kern) as full, make_solver(w, kernel=kern) as first:
        full.run(0, w.nt)
        full.synchronize()
        first.run(0, k)
        path = str(tmp_path / "state.ckpt")
        blob = first.checkpoint(k, path if via == "file" else None)
        if via == "file":
            assert os.path.getsize(path) == first.checkpoint_bytes()
            blob = open(path, "rb").read()
        hd = sgfd.checkpoint_header(blob)
        assert (hd["nx"], hd["ny"], hd["nz"], hd["pml"], hd["it_next"]) == (w.cfg["nx"], w.cfg["ny"], w.cfg["nz"],
                                                                           w.cfg["pml"], k)
        assert hd["payload_bytes"] + 128 == len(blob)
        assert sgfd.checkpoint_checksum(blob[128:]) == hd["checksum"]
        # the first handle keeps going after a checkpoint, unaffected
        first.run(k, w.nt - k)
        np.testing.assert_array_equal(first.traces(), full.traces())
    with make_solver(w, kernel=kern) as resumed:
        it_next = resumed.restore(path if via == "file" else blob)
        assert it_next == k
        resumed.run(it_next, w.nt - it_next)
        resumed.synchronize()
        ref = make_solver(w, kernel=kern)
        ref.run(0, w.nt)
        np.testing.assert_array_equal(resumed.traces(), ref.traces())
        for fid in range(9):
            np.testing.assert_array_equal(resumed.field(fid), ref.field(fid), err_msg=sgfd.FIELD_NAMES[fid])
        ref.close()


def test_checkpoint_rejects_mismatch_and_corruption(tmp_path):
    w = wl.small_random_case(nt=30)
    with make_solver(w) as s:
        s.run(0, 20)
        blob = bytearray(s.checkpoint(20))
    other = wl.small_random_case(nx=39, nt=30)
    with make_solver(other) as s:
        with pytest.raises(sgfd.SgfdError) as e:
            s.restore(bytes(blob))
        assert e.value.code == sgfd.ERR_INVALID and "grid" in str(e.value)
    with make_solver(w) as s:
        s.run(0, 5)
        bad = bytearray(blob)
        bad[128 + len(bad) // 3] ^= 0x40
        with pytest.raises(sgfd.SgfdError) as e:
            s.restore(bytes(bad))
        assert "checksum" in str(e.value)
        for fid in range(9):   # a failed load leaves zeros, not a half-loaded state
            assert not s.field(fid).any()
        with pytest.raises(sgfd.SgfdError):
            s.restore(bytes(blob[:-7]))
        with pytest.raises(sgfd.SgfdError):
            s.restore(b"NOTACKPT" + bytes(blob[8:]))
        with pytest.raises(sgfd.SgfdError):
            s.restore(str(tmp_path / "missing.ckpt"))


def test_station_files(tmp_path):
    w = wl.small_random_case(nt=40, nrec=24)
    with make_solver(w) as s:
        s.run(0, w.nt)
        tr = s.traces()
        prefix = str(tmp_path / "shot")
        s.write_stations(prefix)
        table = np.loadtxt(prefix + "_receivers.txt", dtype=str)
        assert len(table) == len(w.rec_comp)
        names = ["vx", "vy", "vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"]
        for c in sorted(set(w.rec_comp.tolist())):
            members = np.flatnonzero(w.rec_comp == c)
            txt = np.loadtxt(prefix + f"_{names[c]}.txt", ndmin=2)
            assert txt.shape == (w.nt, len(members))
            # %g keeps 6 significant digits; compare in float64 so that the
            # tolerance of subnormal samples does not underflow
            np.testing.assert_allclose(txt, tr[members].T.astype(np.float64), rtol=1e-5, atol=0)
            raw = np.fromfile(prefix + f"_{names[c]}.bin", dtype=np.int32, count=2)
            assert tuple(raw) == (w.nt, len(members))
            binv = np.fromfile(prefix + f"_{names[c]}.bin", dtype=np.float32, offset=8).reshape(w.nt, -1)
            np.testing.assert_array_equal(binv, tr[members].T)
            assert (table[members, 4] == names[c]).all()
            assert (table[members, 5].astype(int) == np.arange(len(members))).all()
        for c in set(range(9)) - set(w.rec_comp.tolist()):
            assert not os.path.exists(prefix + f"_{names[c]}.txt")
        s.write_stations(prefix + "_short", nsteps=10, binary=False)
        c0 = int(w.rec_comp[0])
        assert np.loadtxt(prefix + f"_short_{names[c0]}.txt", ndmin=2).shape[0] == 10
        assert not os.path.exists(prefix + f"_short_{names[c0]}.bin")


def test_trace_range_readback():
    """sgfd_get_trace_range: one time-major block of steps equals the same
    steps of sgfd_get_traces and of sgfd_get_trace_step; ranges past the
    trace length are rejected."""
    w = wl.small_random_case(nt=40, nrec=24)
    with make_solver(w) as s:
        for it in range(25):
            s.step(it, float(w.wavelet[it]))
        block = s.trace_range(3, 20)
        tr = s.traces()
        np.testing.assert_array_equal(block, tr[:, 3:23].T)
        np.testing.assert_array_equal(block[5], s.trace_step(8))
        assert s.trace_range(0, 0).shape == (0, len(w.rec_comp))
        with pytest.raises(sgfd.SgfdError):
            s.trace_range(30, 11)


def test_checkpoint_moves_between_kernel_families():
    """The checkpoint layout does not depend on the kernel family: a state saved
    by the z-marching kernels resumes on the per-cell kernels bit for bit."""
    w = wl.small_random_case(nt=50)
    with make_solver(w) as full:
        full.run(0, w.nt)
        tr = full.traces()
    with make_solver(w, kernel=sgfd.KERNEL_ZMARCH) as a:
        a.run(0, 23)
        blob = a.checkpoint(23)
    with make_solver(w, kernel=sgfd.KERNEL_SIMPLE) as b:
        b.run(b.restore(blob), w.nt - 23)
        np.testing.assert_array_equal(b.traces(), tr)

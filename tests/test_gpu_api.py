"""Behaviour of the C ABI on a GPU: state errors, argument checks, reset,
receivers on the frame, per-step readback and profiling."""
import numpy as np
import pytest

from helpers import make_solver, run_oracle
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu


def test_step_before_medium_is_a_state_error():
    s = sgfd.Solver(sgfd.default_config(nx=30, ny=30, nz=30, pml=4))
    with pytest.raises(sgfd.SgfdError) as e:
        s.step(0, 1.0)
    assert e.value.code == sgfd.ERR_STATE
    s.close()


def test_bad_source_and_receivers_rejected():
    s = sgfd.Solver(sgfd.default_config(nx=30, ny=30, nz=30, pml=4))
    for xyz in ((4, 10, 10), (10, 25, 10), (-1, 3, 3)):
        with pytest.raises(sgfd.SgfdError) as e:
            s.set_source(*xyz)
        assert e.value.code == sgfd.ERR_INVALID
    with pytest.raises(sgfd.SgfdError):
        s.set_receivers([[30, 0, 0]], [0], 10)
    with pytest.raises(sgfd.SgfdError):
        s.set_receivers([[3, 3, 3]], [9], 10)
    s.close()


def test_reset_reproduces_run_and_frame_receivers_stay_zero():
    w = wl.small_random_case(nt=30)
    w.rec_xyz = np.concatenate([w.rec_xyz, [[0, 0, 0], [2, 3, 4]]]).astype(np.int32)
    w.rec_comp = np.concatenate([w.rec_comp, [sgfd.TXX, sgfd.VX]]).astype(np.int32)
    with make_solver(w) as s:
        s.run(0, w.nt)
        a = s.traces()
        s.reset()
        s.run(0, w.nt)
        b = s.traces()
        np.testing.assert_array_equal(a, b)
        assert np.all(a[-2:] == 0)
        # per-step readback equals the column of the full trace
        np.testing.assert_array_equal(s.trace_step(17), a[:, 17])


def test_profile_runs_and_matches_plain_run():
    w = wl.small_random_case(nt=20)
    o = run_oracle(w)
    with make_solver(w) as s:
        tv, ts = s.profile(0, w.nt)
        assert tv > 0 and ts > 0
        np.testing.assert_array_equal(s.traces(), o.traces().astype(np.float32))


def test_cell_counts():
    w = wl.plain_cube(n_interior=20, pml=5, nt=2)
    with make_solver(w) as s:
        ni, npml = s.cell_counts()
        assert ni == 20 ** 3 and ni + npml == 30 ** 3

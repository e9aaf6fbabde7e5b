"""The GPU path against the reference's shipped station trace (1500 steps of
the reference driver's configuration, 3DGPUwithPML_1DArraySingleGPU_concise/
main.cu:11-56 → stationData.txt).  Tolerance: relative L2 1e-5 (the golden is
printed with 6 significant digits)."""
import numpy as np
import pytest

import os

from conftest import ROOT, rel_l2
from helpers import make_solver
import sgfd
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fp64_trace():
    return np.load(os.path.join(ROOT, "tests", "golden", "fp64_trace_reference_main.npy"))


@pytest.mark.parametrize("arith", [sgfd.ARITH_REF, sgfd.ARITH_FAST], ids=["ref", "fast"])
@pytest.mark.parametrize("kernel", [sgfd.KERNEL_SIMPLE, sgfd.KERNEL_ZMARCH], ids=["simple", "zmarch"])
def test_reference_station_trace(golden_trace, fp64_trace, kernel, arith):
    """REF rounding reproduces the reference's FP32 trace within 1e-5.  Both
    rounding modes are within 1e-5 of exact (FP64) arithmetic — the reference's
    own trace is 8.2e-6 from it — and FAST, a different FP32 rounding, is
    within 1.5e-5 of the reference's trace (two FP32 roundings of this
    1500-step run differ by about sqrt(2) x 8e-6)."""
    w = wl.reference_case(nt=1500)
    with make_solver(w, kernel=kernel, arith=arith) as s:
        s.run(0, w.nt)
        tr = s.traces()[0].astype(np.float64)
    err = rel_l2(tr, golden_trace)
    assert err < (1e-5 if arith == sgfd.ARITH_REF else 1.5e-5), err
    assert rel_l2(tr, fp64_trace) < 1e-5
    assert np.argmax(tr) == np.argmax(golden_trace) == 235
    # the late coda (PML reflections ~1e-12..1e-15) is reproduced too
    late = slice(1000, 1500)
    assert rel_l2(tr[late], golden_trace[late]) < 1e-3
    # first arrival of the precursor at the same step as the golden
    assert np.nonzero(tr)[0][0] == np.nonzero(golden_trace)[0][0] == 10

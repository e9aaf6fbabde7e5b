"""The GPU path against the reference's shipped station trace (1500 steps of
the reference driver's configuration, 3DGPUwithPML_1DArraySingleGPU_concise/
main.cu:11-56 → stationData.txt).  Tolerance: relative L2 1e-5 (the golden is
printed with 6 significant digits)."""
import numpy as np
import pytest

from conftest import rel_l2
from helpers import make_solver
import sgfd.workloads as wl

pytestmark = pytest.mark.gpu


def test_reference_station_trace(golden_trace):
    w = wl.reference_case(nt=1500)
    with make_solver(w) as s:
        s.run(0, w.nt)
        tr = s.traces()[0].astype(np.float64)
    err = rel_l2(tr, golden_trace)
    assert err < 1e-5, err
    assert np.argmax(tr) == np.argmax(golden_trace) == 235
    # the late coda (PML reflections ~1e-12..1e-15) is reproduced too
    late = slice(1000, 1500)
    assert rel_l2(tr[late], golden_trace[late]) < 1e-3
    # first arrival of the precursor at the same step as the golden
    assert np.nonzero(tr)[0][0] == np.nonzero(golden_trace)[0][0] == 10

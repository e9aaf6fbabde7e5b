"""Pins the CPU oracle to the reference's only known-answer vector.

tests/golden/stationData_reference_main.txt is the reference's shipped
3DGPUwithPML_1DArraySingleGPU_concise/stationData.txt: the txx station trace
of that directory's main.cu:11-56 configuration (300x200x100 GRID, pml 10,
1500 steps), printed with 6 significant digits by stationDataOutput()
(3DGPUwithPML_1DArraySingleGPU_optimization/ElasticWaveEquation.cu:950-960).
"""
import hashlib
import os

import numpy as np
import pytest

from conftest import ROOT, rel_l2
from helpers import run_oracle
import oracle_py
import sgfd.workloads as wl


def test_golden_fixture_integrity():
    path = os.path.join(ROOT, "tests", "golden", "stationData_reference_main.txt")
    want = open(path + ".sha256").read().split()[0]
    assert hashlib.sha256(open(path, "rb").read()).hexdigest() == want


def test_oracle_ricker_matches_reference_formula():
    # s(it) of OPT/ElasticWaveEquation.cu:184-189, evaluated independently in float64
    # from the same float32 operands; agreement to float32 rounding.
    f0, dt = np.float32(20.0), np.float32(0.0005)
    w = oracle_py.ricker_ref(20.0, 0.0005, 400)
    t0 = np.ceil(np.float32(1.0) / (f0 * dt))
    it = np.arange(400, dtype=np.float32)
    a = np.float32(3.1415926) * f0 * ((it - t0) * dt - np.float32(1.0) / f0)
    ref = (1 - 2 * a.astype(np.float64) ** 2) * np.exp(-(a.astype(np.float64) ** 2))
    assert np.max(np.abs(w - ref)) < 2e-7


def test_oracle_golden_precursor_exact(golden_trace):
    """First 40 steps with IEEE subnormals.  The precursor samples (1e-37..1e-26,
    golden lines 11-40) start at the same step and agree to the golden's printed
    digits; the reference leaves FMA contraction to nvcc, so a few samples that
    carry cancellation differ in the 5th digit (observed max 3.4e-5)."""
    w = wl.reference_case(nt=40)
    tr = run_oracle(w).traces()[0]
    g = golden_trace[:40]
    assert np.array_equal(np.nonzero(tr)[0], np.nonzero(g)[0])
    nz = g != 0
    rel = np.abs(tr[nz] - g[nz]) / np.abs(g[nz])
    assert np.median(rel) < 2e-6, np.median(rel)
    assert rel.max() < 1e-4, rel.max()


def test_oracle_golden_main_arrival(golden_trace):
    """Steps 0..299 (direct arrival peaks at step 235) with flush-to-zero for
    speed: relative L2 over the trace within the golden's 6-digit rounding."""
    n = 300
    w = wl.reference_case(nt=n)
    tr = run_oracle(w, ftz=True).traces()[0]
    g = golden_trace[:n]
    err = rel_l2(tr, g)
    assert err < 1e-5, err
    assert abs(np.argmax(tr) - np.argmax(g)) == 0


def test_fp64_fixture_against_reference_trace(golden_trace):
    """The committed FP64 oracle trace (tests/golden/make_fp64_trace.py) sits
    within FP32 rounding of the reference's own trace: 8.2e-6 relative L2."""
    d64 = np.load(os.path.join(ROOT, "tests", "golden", "fp64_trace_reference_main.npy"))
    assert d64.shape == golden_trace.shape
    assert rel_l2(golden_trace, d64) < 1e-5
    assert np.argmax(d64) == np.argmax(golden_trace)

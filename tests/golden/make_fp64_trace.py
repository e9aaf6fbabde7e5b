"""FP64 oracle station trace of the reference driver's configuration.

Runs the CPU oracle (oracle/, REF rounding, float64 arithmetic) on the
configuration of 3DGPUwithPML_1DArraySingleGPU_concise/main.cu:11-56 for
1500 steps and saves the txx station trace.  GPU tests compare both rounding
modes against it ("error against exact arithmetic"); the reference's own FP32
trace (stationData_reference_main.txt) is 8.2e-6 relative L2 away from it.

Usage: python tests/golden/make_fp64_trace.py     (about 2 minutes on 8 cores)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "staggered-grid_b200"), os.path.join(ROOT, "oracle")]

from helpers import run_oracle  # noqa: E402
import sgfd.workloads as wl     # noqa: E402


def main():
    w = wl.reference_case(nt=1500)
    tr = run_oracle(w, fp64=True, ftz=True).traces()[0]
    np.save(os.path.join(HERE, "fp64_trace_reference_main.npy"), tr)
    print("saved", tr.shape, float(np.abs(tr).max()))


if __name__ == "__main__":
    main()

"""Copies the reference's known-answer station trace into tests/golden/.

The reference ships one golden vector for the hot path:
3DGPUwithPML_1DArraySingleGPU_concise/stationData.txt, the txx trace of 1500
steps written by stationDataOutput() (…/ElasticWaveEquation.cu, one value per
line, 6 significant digits) for the configuration of that directory's
main.cu:11-56.  The reference tree is not available where GPU tests run, so a
verbatim copy is kept here with its SHA-256.

Usage: python tests/golden/make_golden.py [/path/to/reference]
(default: $SGFD_REFERENCE_DIR, else /root/reference)
"""
import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = "3DGPUwithPML_1DArraySingleGPU_concise/stationData.txt"
DST = os.path.join(HERE, "stationData_reference_main.txt")


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SGFD_REFERENCE_DIR", "/root/reference")
    shutil.copyfile(os.path.join(ref, SRC), DST)
    digest = hashlib.sha256(open(DST, "rb").read()).hexdigest()
    with open(DST + ".sha256", "w") as f:
        f.write(f"{digest}  {os.path.basename(DST)}\n")
    print(digest)


if __name__ == "__main__":
    main()

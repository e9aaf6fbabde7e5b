"""ctypes binding of the CPU oracle (oracle/libsgfd_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, as the checker.  The product never imports it.

The oracle restates the reference's single-GPU PML timestep loop
(3DGPUwithPML_1DArraySingleGPU_optimization/ElasticWaveEquation.cu:191-841);
see oracle/sgfd_oracle.cpp for the algorithm and its citations.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libsgfd_oracle.so")
_lib = None


class OracleConfig(ctypes.Structure):
    """Mirror of sgfd_config (include/sgfd.h)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("pml", ctypes.c_int32),
        ("dt", ctypes.c_float), ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
        ("coef", ctypes.c_float * 5),
        ("damping", ctypes.c_int32), ("damping_R", ctypes.c_float), ("damping_vconst", ctypes.c_float),
        ("quirks", ctypes.c_int32), ("storage", ctypes.c_int32), ("kernel", ctypes.c_int32),
        ("device", ctypes.c_int32), ("arith", ctypes.c_int32), ("reserved", ctypes.c_int32 * 7),
    ]


def build():
    """Compile the oracle library with oracle/Makefile (needs g++ with OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "libsgfd_oracle.so"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.sgo_create.restype = ctypes.c_void_p
        L.sgo_create.argtypes = [ctypes.POINTER(OracleConfig), ctypes.c_int]
        L.sgo_destroy.argtypes = [ctypes.c_void_p]
        L.sgo_set_threads.argtypes = [ctypes.c_int]
        L.sgo_set_ftz.argtypes = [ctypes.c_void_p, ctypes.c_int]
        fp = ctypes.POINTER(ctypes.c_float)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int32)
        L.sgo_set_medium.argtypes = [ctypes.c_void_p, fp, fp, fp]
        L.sgo_set_source.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.sgo_set_receivers.argtypes = [ctypes.c_void_p, ctypes.c_int, ip, ip, ctypes.c_int]
        L.sgo_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, dp]
        L.sgo_get_traces.argtypes = [ctypes.c_void_p, dp]
        L.sgo_get_field.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.sgo_set_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
        L.sgo_round16.argtypes = [ctypes.c_int, fp, fp, ctypes.c_int64]
        L.sgo_scale_exponents.argtypes = [ctypes.c_void_p, ip]
        L.sgo_ricker_ref.restype = ctypes.c_float
        L.sgo_ricker_ref.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def set_threads(n: int) -> int:
    return lib().sgo_set_threads(int(n))


def round16(storage: int, x) -> np.ndarray:
    """The oracle's 16-bit rounding (storage 1 = bfloat16, 2 = binary16), as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty_like(x)
    lib().sgo_round16(int(storage), _ptr(x, ctypes.c_float), _ptr(out, ctypes.c_float), x.size)
    return out


def ricker_ref(f0: float, dt: float, nt: int) -> np.ndarray:
    """Reference wavelet values (float32) for it = 0..nt-1."""
    L = lib()
    return np.array([L.sgo_ricker_ref(f0, dt, it) for it in range(nt)], dtype=np.float32)


class Oracle:
    """One oracle model; mirrors the product handle's call sequence."""

    def __init__(self, cfg: dict, fp64: bool = False, ftz: bool = False):
        c = OracleConfig()
        for k, v in cfg.items():
            if k == "coef":
                for i in range(5):
                    c.coef[i] = float(v[i])
            elif hasattr(c, k):
                setattr(c, k, v)
        self.cfg = c
        self.shape = (c.nz, c.ny, c.nx)
        self.h = lib().sgo_create(ctypes.byref(c), 1 if fp64 else 0)
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        if ftz:
            lib().sgo_set_ftz(self.h, 1)
        self.nrec = 0
        self.nt = 0

    def close(self):
        if self.h:
            lib().sgo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_medium(self, b, lam, mu):
        b = np.ascontiguousarray(b, dtype=np.float32)
        lam = np.ascontiguousarray(lam, dtype=np.float32)
        mu = np.ascontiguousarray(mu, dtype=np.float32)
        assert b.size == lam.size == mu.size == int(np.prod(self.shape))
        lib().sgo_set_medium(self.h, _ptr(b, ctypes.c_float), _ptr(lam, ctypes.c_float), _ptr(mu, ctypes.c_float))

    def set_source(self, x, y, z):
        if lib().sgo_set_source(self.h, x, y, z) != 0:
            raise ValueError("source outside the computed region")

    def set_receivers(self, xyz, comp, nt):
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        comp = np.ascontiguousarray(np.asarray(comp, dtype=np.int32).reshape(-1))
        if lib().sgo_set_receivers(self.h, len(comp), _ptr(xyz, ctypes.c_int32), _ptr(comp, ctypes.c_int32), nt) != 0:
            raise ValueError("bad receivers")
        self.nrec, self.nt = len(comp), nt

    def run(self, wavelet, it0=0, nsteps=None):
        w = np.ascontiguousarray(np.asarray(wavelet, dtype=np.float64))
        if nsteps is None:
            nsteps = len(w) - it0
        assert it0 + nsteps <= len(w)
        lib().sgo_run(self.h, it0, nsteps, _ptr(w, ctypes.c_double))

    def traces(self) -> np.ndarray:
        out = np.zeros((self.nrec, self.nt), dtype=np.float64)
        lib().sgo_get_traces(self.h, _ptr(out, ctypes.c_double))
        return out

    def scale_exponents(self) -> np.ndarray:
        """Per-field scale exponents of the 16-bit storage emulation."""
        out = np.zeros(9, dtype=np.int32)
        lib().sgo_scale_exponents(self.h, _ptr(out, ctypes.c_int32))
        return out

    def field(self, fid: int) -> np.ndarray:
        out = np.zeros(self.shape, dtype=np.float64)
        lib().sgo_get_field(self.h, int(fid), _ptr(out, ctypes.c_double))
        return out

    def set_field(self, fid: int, values):
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(self.shape))
        if lib().sgo_set_field(self.h, int(fid), _ptr(a, ctypes.c_float)) != 0:
            raise ValueError("bad field")


# ---------------------------------------------------------------------------
# The reference's own GPU program (oracle/_ref/ref_opt, built by oracle/Makefile
# from 3DGPUwithPML_1DArraySingleGPU_optimization/ElasticWaveEquation.cu).
# ---------------------------------------------------------------------------

REF_OPT = os.path.join(_HERE, "_ref", "ref_opt")
DROPIN_MAIN = os.path.join(_HERE, "_ref", "dropin_main")


def write_ref_case(path, cfg: dict, b, lam, mu, src, station, nt: int, f0: float):
    """Case file for ref_opt (format documented in oracle/ref_harness.cu)."""
    with open(path, "wb") as f:
        hdr = np.array([0x43464753, 1, cfg["nx"], cfg["ny"], cfg["nz"], cfg["pml"], nt, *src, *station, 0], np.int32)
        f.write(hdr.tobytes())
        fl = np.array([cfg["dt"], cfg["dx"], cfg["dy"], cfg["dz"], f0, *cfg["coef"]], np.float32)
        f.write(fl.tobytes())
        for a in (b, lam, mu):
            f.write(np.ascontiguousarray(a, np.float32).tobytes())


def run_ref_opt(workdir, cfg: dict, b, lam, mu, src, station, nt: int, f0: float):
    """Run the reference program; returns (station trace [nt], fields [9, nz, ny, nx], device ms)."""
    case = os.path.join(workdir, "case.bin")
    out = os.path.join(workdir, "out.bin")
    write_ref_case(case, cfg, b, lam, mu, src, station, nt, f0)
    r = subprocess.run([REF_OPT, case, out], capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        raise RuntimeError(f"ref_opt failed: {r.stderr[-500:]}")
    ms = float(r.stdout.split("ms=")[1].split()[0])
    data = np.fromfile(out, dtype=np.float32)
    n = cfg["nx"] * cfg["ny"] * cfg["nz"]
    trace = data[:nt]
    fields = data[nt:].reshape(9, cfg["nz"], cfg["ny"], cfg["nx"])
    return trace, fields, ms

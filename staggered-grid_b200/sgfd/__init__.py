"""Python binding of libsgfd.so (include/sgfd.h) for tests, benchmarks and scripting.

The product is the C ABI and its CUDA kernels; this module is a thin ctypes
layer over it.  There is no CPU code path: if the shared library is missing
or no CUDA device is present, creating a Solver raises.

Typical use (mirrors the reference driver 3DGPUwithPML_1DArraySingleGPU_concise/main.cu:11-79):

    cfg = sgfd.default_config(nx=300, ny=200, nz=100, pml=10, dt=5e-4)
    s = sgfd.Solver(cfg)
    s.set_medium(b, lam, mu)               # float32 arrays of nx*ny*nz, x fastest
    s.set_source(150, 100, 50)
    s.set_receivers([[160, 110, 60]], [sgfd.TXX], nt=1500)
    s.set_wavelet(sgfd.ricker_ref(20.0, 5e-4, 1500))
    s.run(0, 1500); s.synchronize()
    trace = s.traces()[0]
"""
from __future__ import annotations

import ctypes
import struct
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_PKG), "lib", "libsgfd.so")

VX, VY, VZ, TXX, TYY, TZZ, TXY, TXZ, TYZ = range(9)
FIELD_NAMES = ["vx", "vy", "vz", "txx", "tyy", "tzz", "txy", "txz", "tyz"]
BUOYANCY, LAMBDA, MU = range(3)
DAMP_REFGPU, DAMP_LOGR, DAMP_REFCPU = range(3)
QUIRKS_REF, QUIRKS_FIXED = range(2)
STORE_F32, STORE_BF16, STORE_F16 = range(3)
KERNEL_AUTO, KERNEL_SIMPLE, KERNEL_ZMARCH = range(3)
ARITH_REF, ARITH_FAST = range(2)
REGION_COMPUTED, REGION_INTERIOR, REGION_PML = range(3)
HALO_LOW, HALO_HIGH = range(2)             # the cut below / above a z-slab
HALO_STRESS, HALO_VELOCITY = range(2)      # txz, tyz, tzz / vx, vy, vz
PHASE_VELOCITY, PHASE_STRESS = range(2)
PART_INNER, PART_OUTER = 1, 2              # planes that read no frame plane / the rest

# sgfd_status
OK, ERR_INVALID, ERR_ALLOC, ERR_CUDA, ERR_STATE, ERR_UNSUPPORTED, ERR_NO_DEVICE, ERR_NONFINITE = range(8)

REF_COEF = (1.21124, -8.97217e-2, 1.38428e-2, -1.76566e-3, 1.18680e-4)


class Config(ctypes.Structure):
    """sgfd_config (include/sgfd.h)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("pml", ctypes.c_int32),
        ("dt", ctypes.c_float), ("dx", ctypes.c_float), ("dy", ctypes.c_float), ("dz", ctypes.c_float),
        ("coef", ctypes.c_float * 5),
        ("damping", ctypes.c_int32), ("damping_R", ctypes.c_float), ("damping_vconst", ctypes.c_float),
        ("quirks", ctypes.c_int32), ("storage", ctypes.c_int32), ("kernel", ctypes.c_int32),
        ("device", ctypes.c_int32), ("arith", ctypes.c_int32), ("nz_total", ctypes.c_int32),
        ("z_offset", ctypes.c_int32), ("reserved", ctypes.c_int32 * 5),
    ]


class SgfdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sgfd error {code}: {msg}")
        self.code = code


class Tuning(ctypes.Structure):
    """sgfd_tuning: the launch shape sgfd_autotune picked."""
    _fields_ = [("kernel", ctypes.c_int32), ("tile_rows", ctypes.c_int32), ("zchunk", ctypes.c_int32),
                ("candidates", ctypes.c_int32), ("ms_per_step", ctypes.c_float), ("tile_cols", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 2)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libsgfd.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C staggered-grid_b200` "
                          "or __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    vp, fp, ip = ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int32)
    i32 = ctypes.c_int32
    sigs = {
        "sgfd_abi_version": (ctypes.c_int, []),
        "sgfd_config_default": (None, [ctypes.POINTER(Config)]),
        "sgfd_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(vp)]),
        "sgfd_destroy": (None, [vp]),
        "sgfd_last_error": (ctypes.c_char_p, [vp]),
        "sgfd_global_error": (ctypes.c_char_p, []),
        "sgfd_set_stream": (ctypes.c_int, [vp, vp]),
        "sgfd_set_medium": (ctypes.c_int, [vp, fp, fp, fp]),
        "sgfd_set_medium_device": (ctypes.c_int, [vp, vp, vp, vp]),
        "sgfd_set_source": (ctypes.c_int, [vp, i32, i32, i32]),
        "sgfd_set_receivers": (ctypes.c_int, [vp, i32, ip, ip, i32]),
        "sgfd_set_wavelet": (ctypes.c_int, [vp, i32, fp]),
        "sgfd_step": (ctypes.c_int, [vp, i32, ctypes.c_float]),
        "sgfd_step_phase": (ctypes.c_int, [vp, i32, ctypes.c_float, i32]),
        "sgfd_step_phase_part": (ctypes.c_int, [vp, i32, ctypes.c_float, i32, i32]),
        "sgfd_halo_bytes": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int64)]),
        "sgfd_halo_pack": (ctypes.c_int, [vp, i32, i32, vp]),
        "sgfd_halo_unpack": (ctypes.c_int, [vp, i32, i32, vp]),
        "sgfd_run": (ctypes.c_int, [vp, i32, i32, i32]),
        "sgfd_synchronize": (ctypes.c_int, [vp]),
        "sgfd_reset": (ctypes.c_int, [vp]),
        "sgfd_get_traces": (ctypes.c_int, [vp, fp]),
        "sgfd_get_trace_range": (ctypes.c_int, [vp, i32, i32, fp]),
        "sgfd_get_trace_step": (ctypes.c_int, [vp, i32, fp]),
        "sgfd_profile": (ctypes.c_int, [vp, i32, i32, fp, fp]),
        "sgfd_get_field": (ctypes.c_int, [vp, i32, fp]),
        "sgfd_set_field": (ctypes.c_int, [vp, i32, fp]),
        "sgfd_get_medium": (ctypes.c_int, [vp, i32, fp]),
        "sgfd_ricker_ref": (ctypes.c_float, [ctypes.c_float, ctypes.c_float, i32]),
        "sgfd_ricker_t0": (ctypes.c_float, [ctypes.c_float, ctypes.c_float, ctypes.c_float, i32]),
        "sgfd_set_zchunk": (ctypes.c_int, [vp, i32]),
        "sgfd_set_tiling": (ctypes.c_int, [vp, i32, i32]),
        "sgfd_cell_counts": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
        "sgfd_launches_per_step": (ctypes.c_int, [vp]),
        "sgfd_set_tile": (ctypes.c_int, [vp, i32, i32, i32]),
        "sgfd_get_tile": (ctypes.c_int, [vp, ip, ip, ip]),
        "sgfd_device_allocations": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int64)]),
        "sgfd_run_launches": (ctypes.c_int, [vp, ctypes.c_int32, ctypes.c_int32]),
        "sgfd_prepare_run": (ctypes.c_int, [vp]),
        "sgfd_kernel_name": (ctypes.c_char_p, [vp]),
        "sgfd_checkpoint_bytes": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int64)]),
        "sgfd_checkpoint_save": (ctypes.c_int, [vp, i32, vp, ctypes.c_int64]),
        "sgfd_checkpoint_load": (ctypes.c_int, [vp, vp, ctypes.c_int64, ip]),
        "sgfd_checkpoint_write": (ctypes.c_int, [vp, i32, ctypes.c_char_p]),
        "sgfd_checkpoint_read": (ctypes.c_int, [vp, ctypes.c_char_p, ip]),
        "sgfd_write_stations": (ctypes.c_int, [vp, ctypes.c_char_p, i32, i32]),
        "sgfd_set_kernel": (ctypes.c_int, [vp, i32]),
        "sgfd_autotune": (ctypes.c_int, [vp, i32, ctypes.POINTER(Tuning)]),
        "sgfd_batch_create": (ctypes.c_int, [ctypes.POINTER(vp), i32, ctypes.POINTER(vp)]),
        "sgfd_batch_destroy": (None, [vp]),
        "sgfd_batch_last_error": (ctypes.c_char_p, [vp]),
        "sgfd_batch_run": (ctypes.c_int, [vp, i32, i32]),
        "sgfd_batch_synchronize": (ctypes.c_int, [vp]),
        "sgfd_batch_stream": (vp, [vp]),
        "sgfd_batch_run_launches": (ctypes.c_int, [vp, i32]),
        "sgfd_batch_set_persistent": (ctypes.c_int, [vp, i32, i32]),
        "sgfd_set_audit": (ctypes.c_int, [vp, i32, i32, i32]),
        "sgfd_get_audit": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_double)]),
        "sgfd_energy_noalloc": (ctypes.c_int, [vp, i32, i32, ctypes.POINTER(ctypes.c_double),
                                                ctypes.POINTER(ctypes.c_double)]),
        "sgfd_set_learned_strip": (ctypes.c_int, [vp, i32, fp]),
        "sgfd_strip_features": (ctypes.c_int, [vp, i32, i32, ip, fp, fp, fp]),
        "sgfd_copy_window": (ctypes.c_int, [vp, vp, i32, i32, i32]),
        "sgfd_sample_fields": (ctypes.c_int, [vp, i32, ip, fp]),
        "sgfd_mlp_param_count": (ctypes.c_int, []),
        "sgfd_mlp_forward": (ctypes.c_int, [i32, fp, fp, ctypes.c_int64, fp]),
        "sgfd_mlp_infer": (ctypes.c_int, [i32, fp, fp, ctypes.c_int64, fp]),
        "sgfd_mlp_gradient": (ctypes.c_int, [i32, fp, fp, fp, i32, fp, fp]),
        "sgfd_mlp_train": (ctypes.c_int, [i32, fp, fp, fp, ctypes.c_int64, i32, i32, ctypes.c_float, fp]),
        "sgfd_energy": (ctypes.c_int, [vp, i32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def default_config(**kw) -> Config:
    c = Config()
    lib().sgfd_config_default(ctypes.byref(c))
    for k, v in kw.items():
        if k == "coef":
            for i in range(5):
                c.coef[i] = float(v[i])
        elif not hasattr(c, k):
            raise KeyError(k)
        else:
            setattr(c, k, v)
    return c


def config_dict(c: Config) -> dict:
    d = {k: getattr(c, k) for k, _ in Config._fields_ if k not in ("coef", "reserved")}
    d["coef"] = [c.coef[i] for i in range(5)]
    return d


def ricker_ref(f0: float, dt: float, nt: int) -> np.ndarray:
    """Reference Ricker values s(it), it = 0..nt-1 (OPT/ElasticWaveEquation.cu:184-189)."""
    L = lib()
    return np.array([L.sgfd_ricker_ref(f0, dt, i) for i in range(nt)], dtype=np.float32)


def ricker_t0(f0: float, dt: float, t0: float, nt: int) -> np.ndarray:
    L = lib()
    return np.array([L.sgfd_ricker_t0(f0, dt, t0, i) for i in range(nt)], dtype=np.float32)


class Solver:
    """One model on one GPU (an sgfd_solver handle)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.shape = (cfg.nz, cfg.ny, cfg.nx)
        h = ctypes.c_void_p()
        rc = lib().sgfd_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != OK:
            raise SgfdError(rc, lib().sgfd_global_error().decode())
        self.h = h
        self.nrec = 0
        self.nt = 0

    def _check(self, rc: int):
        if rc != OK:
            raise SgfdError(rc, lib().sgfd_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            lib().sgfd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_ptr: int | None):
        self._check(lib().sgfd_set_stream(self.h, stream_ptr))

    def set_medium(self, b, lam, mu):
        arrs = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1) for a in (b, lam, mu)]
        n = int(np.prod(self.shape))
        if any(a.size != n for a in arrs):
            raise ValueError(f"medium arrays must have {n} cells")
        self._check(lib().sgfd_set_medium(self.h, *[_fptr(a) for a in arrs]))

    def set_medium_device(self, b_ptr: int, lam_ptr: int, mu_ptr: int):
        self._check(lib().sgfd_set_medium_device(self.h, b_ptr, lam_ptr, mu_ptr))

    def set_source(self, x: int, y: int, z: int):
        self._check(lib().sgfd_set_source(self.h, x, y, z))

    def set_receivers(self, xyz, comp, nt: int):
        xyz = np.ascontiguousarray(np.asarray(xyz, dtype=np.int32).reshape(-1, 3))
        comp = np.ascontiguousarray(np.asarray(comp, dtype=np.int32).reshape(-1))
        if len(xyz) != len(comp):
            raise ValueError("one component per receiver")
        self._check(lib().sgfd_set_receivers(
            self.h, len(comp), xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            comp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), nt))
        self.nrec, self.nt = len(comp), nt

    def set_wavelet(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(lib().sgfd_set_wavelet(self.h, len(w), _fptr(w)))

    def step(self, it: int, value: float):
        self._check(lib().sgfd_step(self.h, it, value))

    def step_phase(self, it: int, value: float, phase: int, parts: int = PART_INNER | PART_OUTER):
        """Half a step: PHASE_VELOCITY (source, velocity update, velocity
        receivers) or PHASE_STRESS (stress update, stress receivers); parts
        PART_INNER (planes that read no frame plane) then PART_OUTER split it."""
        self._check(lib().sgfd_step_phase_part(self.h, it, value, phase, parts))

    def halo_bytes(self) -> int:
        """Bytes of one halo buffer of a z-slab (3 fields x 5 padded planes)."""
        n = ctypes.c_int64()
        self._check(lib().sgfd_halo_bytes(self.h, ctypes.byref(n)))
        return n.value

    def halo_pack(self, side: int, kind: int, dst_ptr: int):
        """The slab's own 5 planes beside cut `side` to the device buffer at dst_ptr."""
        self._check(lib().sgfd_halo_pack(self.h, side, kind, dst_ptr))

    def halo_unpack(self, side: int, kind: int, src_ptr: int):
        """A received device buffer into the slab's 5 frame planes on `side`."""
        self._check(lib().sgfd_halo_unpack(self.h, side, kind, src_ptr))

    def run(self, it0: int, nsteps: int, graph: bool = True):
        self._check(lib().sgfd_run(self.h, it0, nsteps, 1 if graph else 0))

    def prepare_run(self):
        self._check(lib().sgfd_prepare_run(self.h))

    def synchronize(self):
        self._check(lib().sgfd_synchronize(self.h))

    def reset(self):
        self._check(lib().sgfd_reset(self.h))

    def traces(self) -> np.ndarray:
        out = np.zeros((self.nrec, self.nt), dtype=np.float32)
        if self.nrec:
            self._check(lib().sgfd_get_traces(self.h, _fptr(out)))
        return out

    def trace_range(self, it0: int, n: int, out: np.ndarray | None = None) -> np.ndarray:
        """Samples of steps it0 .. it0+n-1, time-major [n][nrec], in one transfer."""
        if out is None:
            out = np.zeros((n, self.nrec), dtype=np.float32)
        assert out.dtype == np.float32 and out.flags.c_contiguous and out.size >= n * self.nrec
        self._check(lib().sgfd_get_trace_range(self.h, it0, n, _fptr(out)))
        return out

    def trace_step(self, it: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.nrec, dtype=np.float32)
        self._check(lib().sgfd_get_trace_step(self.h, it, _fptr(out)))
        return out

    def profile(self, it0: int, nsteps: int) -> tuple[float, float]:
        """(ms in velocity kernels, ms in stress kernels) over nsteps steps."""
        a, b = ctypes.c_float(), ctypes.c_float()
        self._check(lib().sgfd_profile(self.h, it0, nsteps, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def field(self, fid: int) -> np.ndarray:
        out = np.zeros(self.shape, dtype=np.float32)
        self._check(lib().sgfd_get_field(self.h, fid, _fptr(out)))
        return out

    def set_field(self, fid: int, values):
        a = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        if a.size != int(np.prod(self.shape)):
            raise ValueError("field arrays must have nx*ny*nz cells")
        self._check(lib().sgfd_set_field(self.h, fid, _fptr(a)))

    def medium(self, which: int) -> np.ndarray:
        out = np.zeros(self.shape, dtype=np.float32)
        self._check(lib().sgfd_get_medium(self.h, which, _fptr(out)))
        return out

    def set_zchunk(self, planes: int):
        self._check(lib().sgfd_set_zchunk(self.h, planes))

    def set_tiling(self, tile_rows: int, zchunk: int = 0):
        self._check(lib().sgfd_set_tiling(self.h, tile_rows, zchunk))

    def set_tile(self, tile_cols: int, tile_rows: int = 8, zchunk: int = 0):
        """z-marching tile shape: 32 x 8, 32 x 16 or 64 x 8 (cell pairs on FP32x2)."""
        self._check(lib().sgfd_set_tile(self.h, tile_cols, tile_rows, zchunk))

    def tile(self) -> tuple[int, int, int]:
        """(tile columns, tile rows, z chunk) of the z-marching kernels in use."""
        a, b, c = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(lib().sgfd_get_tile(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def cell_counts(self) -> tuple[int, int]:
        a, b = ctypes.c_int64(), ctypes.c_int64()
        self._check(lib().sgfd_cell_counts(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def device_allocations(self) -> int:
        """Device allocations the handle has made since it was created."""
        n = ctypes.c_int64()
        self._check(lib().sgfd_device_allocations(self.h, ctypes.byref(n)))
        return n.value

    def launches_per_step(self) -> int:
        return lib().sgfd_launches_per_step(self.h)

    def run_launches(self, nsteps: int, graph: bool = True) -> int:
        return lib().sgfd_run_launches(self.h, nsteps, 1 if graph else 0)

    def kernel_name(self) -> str:
        return lib().sgfd_kernel_name(self.h).decode()

    def set_learned_strip(self, width: int, params=None):
        """Make the outer `width` computed cells a learned absorbing strip (pml = 0 models)."""
        p = None if params is None else np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib().sgfd_set_learned_strip(self.h, width, _fptr(p) if p is not None else None))

    def copy_window_from(self, src: "Solver", x0: int, y0: int, z0: int):
        """This model's 9 fields from the window of src at GRID origin (x0, y0, z0),
        frame zeroed (this model: pml = 0)."""
        self._check(lib().sgfd_copy_window(self.h, src.h, x0, y0, z0))

    def sample_fields(self, cells) -> np.ndarray:
        """The 9 fields [n][9] of the listed cells (computed coordinates)."""
        c = np.ascontiguousarray(np.asarray(cells, dtype=np.int32).reshape(-1, 3))
        out = np.zeros((len(c), 9), np.float32)
        self._check(lib().sgfd_sample_fields(self.h, len(c), c.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                             _fptr(out)))
        return out

    def strip_features(self, width: int, cells):
        """(X [n][252], s [n], rho*vp [n]) of the listed strip cells (computed coordinates)."""
        c = np.ascontiguousarray(np.asarray(cells, dtype=np.int32).reshape(-1, 3))
        n = len(c)
        X = np.zeros((n, 252), np.float32)
        sc = np.zeros(n, np.float32)
        zi = np.zeros(n, np.float32)
        self._check(lib().sgfd_strip_features(self.h, width, n, c.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                              _fptr(X), _fptr(sc), _fptr(zi)))
        return X, sc, zi

    def energy_noalloc(self, region: int = 0, nblocks: int = 0) -> tuple[float, float]:
        """energy() for callers that cannot have the library allocate device
        memory: the scratch is a fixed array inside libsgfd.so (at most 2047
        partial-sum blocks).  Calls that overlap on one GPU race on it."""
        k, e = ctypes.c_double(), ctypes.c_double()
        self._check(lib().sgfd_energy_noalloc(self.h, region, nblocks, ctypes.byref(k), ctypes.byref(e)))
        return k.value, e.value

    def set_audit(self, every: int, region: int = 0, nsamples: int = 0):
        """Record the FP64 energy of `region` after every `every`-th step (0 = off)."""
        self._check(lib().sgfd_set_audit(self.h, every, region, nsamples))
        self.audit_samples = nsamples if every else 0

    def audit(self) -> np.ndarray:
        """(nsamples, 2) array of (kinetic, strain) energy, sample k after step k*every."""
        out = np.zeros((self.audit_samples, 2), dtype=np.float64)
        self._check(lib().sgfd_get_audit(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def set_kernel(self, kernel: int):
        self._check(lib().sgfd_set_kernel(self.h, kernel))

    def autotune(self, probe_steps: int = 0) -> Tuning:
        t = Tuning()
        self._check(lib().sgfd_autotune(self.h, probe_steps, ctypes.byref(t)))
        return t

    def energy(self, region: int = 0) -> tuple[float, float]:
        """(kinetic, strain) energy of the current wavefield over a region, FP64 on the GPU."""
        k, e = ctypes.c_double(), ctypes.c_double()
        self._check(lib().sgfd_energy(self.h, region, ctypes.byref(k), ctypes.byref(e)))
        return k.value, e.value

    # ---- checkpoint / resume and station files ----
    def checkpoint_bytes(self) -> int:
        n = ctypes.c_int64()
        self._check(lib().sgfd_checkpoint_bytes(self.h, ctypes.byref(n)))
        return n.value

    def checkpoint(self, it_next: int, path: str | None = None) -> bytes | None:
        """Save the dynamic state; to `path` when given, else return it as bytes."""
        if path is not None:
            self._check(lib().sgfd_checkpoint_write(self.h, it_next, os.fsencode(path)))
            return None
        buf = ctypes.create_string_buffer(self.checkpoint_bytes())
        self._check(lib().sgfd_checkpoint_save(self.h, it_next, buf, len(buf)))
        return buf.raw

    def restore(self, src: str | bytes) -> int:
        """Load a checkpoint (a path or the bytes of checkpoint()); returns it_next."""
        it = ctypes.c_int32()
        if isinstance(src, (bytes, bytearray)):
            buf = ctypes.create_string_buffer(bytes(src), len(src))
            self._check(lib().sgfd_checkpoint_load(self.h, buf, len(src), ctypes.byref(it)))
        else:
            self._check(lib().sgfd_checkpoint_read(self.h, os.fsencode(src), ctypes.byref(it)))
        return it.value

    def write_stations(self, prefix: str, nsteps: int = 0, binary: bool = True):
        self._check(lib().sgfd_write_stations(self.h, os.fsencode(prefix), nsteps, 1 if binary else 0))


CHECKPOINT_MAGIC = b"SGFDCKP1"
_CKPT_HEADER = struct.Struct("<8sII4i3i3i4fqQQ9bB2x2i12x")


def checkpoint_header(data: bytes) -> dict:
    """Decode the 128-byte header of a checkpoint written by Solver.checkpoint."""
    if len(data) < _CKPT_HEADER.size:
        raise ValueError("shorter than a checkpoint header")
    v = _CKPT_HEADER.unpack_from(data)
    if v[0] != CHECKPOINT_MAGIC:
        raise ValueError("not an sgfd checkpoint")
    keys = ("magic", "version", "header_bytes", "nx", "ny", "nz", "pml", "nrec", "nt", "it_next",
            "quirks", "damping", "arith", "dt", "dx", "dy", "dz", "npml", "payload_bytes", "checksum")
    d = dict(zip(keys, v[:20]))
    d["scale_exponents"] = list(v[20:29])
    d["storage"] = v[29]
    d["nz_total"], d["z_offset"] = v[30], v[31]
    return d


def checkpoint_checksum(payload: bytes) -> int:
    """The header's payload checksum: 4 FNV-1a lanes over 64-bit words, a
    byte-wise tail folded into lane 0, then lanes 1..3 folded in."""
    P, M = 0x100000001B3, (1 << 64) - 1
    lanes = [0xCBF29CE484222325, 0x84222325CBF29CE4, 0x9CE484222325CBF2, 0x2325CBF29CE48422]
    whole = len(payload) // 32 * 32
    w = np.frombuffer(payload[:whole], dtype="<u8").reshape(-1, 4)
    for row in w.tolist():
        for k in range(4):
            lanes[k] = ((lanes[k] ^ row[k]) * P) & M
    h = lanes[0]
    for c in payload[whole:]:
        h = ((h ^ c) * P) & M
    for k in range(1, 4):
        h = ((h ^ lanes[k]) * P) & M
    return h


class Batch:
    """Several Solver models advanced together (sgfd_batch_*): one CUDA graph per
    16 steps with every model's kernels in parallel branches, or (set_persistent)
    one persistent launch per run over all models' work items."""

    def __init__(self, models):
        self.models = list(models)
        arr = (ctypes.c_void_p * len(self.models))(*[m.h for m in self.models])
        h = ctypes.c_void_p()
        rc = lib().sgfd_batch_create(arr, len(self.models), ctypes.byref(h))
        if rc != OK:
            raise SgfdError(rc, lib().sgfd_global_error().decode())
        self.h = h

    def _check(self, rc: int):
        if rc != OK:
            raise SgfdError(rc, lib().sgfd_batch_last_error(self.h).decode())

    def run(self, it0: int, nsteps: int):
        self._check(lib().sgfd_batch_run(self.h, it0, nsteps))

    def set_persistent(self, on: bool = True, barrier_ctas: int = 0):
        """One cooperative launch per run over every model's (tile, z chunk)
        work items, with a bounded grid barrier between the velocity and stress
        phases (barrier_ctas: arrivals each barrier waits for, 0 = launched)."""
        self._check(lib().sgfd_batch_set_persistent(self.h, 1 if on else 0, barrier_ctas))

    def synchronize(self):
        self._check(lib().sgfd_batch_synchronize(self.h))

    def stream(self) -> int:
        return lib().sgfd_batch_stream(self.h) or 0

    def run_launches(self, nsteps: int) -> int:
        return lib().sgfd_batch_run_launches(self.h, nsteps)

    def close(self):
        if getattr(self, "h", None):
            lib().sgfd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# ---- the strip MLP on the GPU (host arrays in and out) ----
MLP_PARAMS = 20937


def _check_global(rc: int):
    if rc != OK:
        raise SgfdError(rc, lib().sgfd_global_error().decode())


def mlp_forward(params, X, device: int = 0) -> np.ndarray:
    p = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    out = np.zeros((len(X), 9), np.float32)
    _check_global(lib().sgfd_mlp_forward(device, _fptr(p), _fptr(X), len(X), _fptr(out)))
    return out


def mlp_infer(params, X, device: int = 0) -> np.ndarray:
    """The strip's tensor-core inference (FP16 operands, FP32 accumulation) on rows X."""
    p = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    out = np.zeros((len(X), 9), np.float32)
    _check_global(lib().sgfd_mlp_infer(device, _fptr(p), _fptr(X), len(X), _fptr(out)))
    return out


def mlp_gradient(params, X, Y, device: int = 0):
    """(loss, gradient) of the mean squared error of the MLP on rows X against Y."""
    p = np.ascontiguousarray(params, np.float32)
    X = np.ascontiguousarray(X, np.float32)
    Y = np.ascontiguousarray(Y, np.float32)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = ctypes.c_float()
    _check_global(lib().sgfd_mlp_gradient(device, _fptr(p), _fptr(X), _fptr(Y), len(X),
                                          ctypes.pointer(loss), _fptr(g)))
    return loss.value, g


def mlp_train(params, X, Y, epochs: int, batch: int = 4096, lr: float = 1e-3, device: int = 0):
    """Minibatch Adam on the GPU; returns (params, per-epoch mean loss)."""
    p = np.ascontiguousarray(params, np.float32).copy()
    X = np.ascontiguousarray(X, np.float32)
    Y = np.ascontiguousarray(Y, np.float32)
    hist = np.zeros(epochs, np.float32)
    _check_global(lib().sgfd_mlp_train(device, _fptr(p), _fptr(X), _fptr(Y), len(X), epochs, batch, lr,
                                       _fptr(hist)))
    return p, hist

"""Workload builders: grids, media, sources, receivers and wavelets.

Each builder returns a `Workload` holding everything a Solver (or the CPU
oracle) needs.  Sizes follow the reference GRID convention (5-cell frame
included on every side).

* `reference_case()` — the reference driver's configuration
  (3DGPUwithPML_1DArraySingleGPU_concise/main.cu:11-56), whose station trace
  ships as CON/stationData.txt.
* `plain_cube()` — homogeneous cube, interior n^3 + PML (configuration
  "plain method, CPU-runnable": 100^3 + 20-cell PML, 101 vx/vz receivers).
* `random_cube()` — random-medium cube (configuration "plain method on GPU":
  344^3 + 20-cell PML, 64x64 receivers recording vx, vy, vz).
* `batch_specs()` / `layered_model()` — the batched configuration: 32
  models of uneven cubic interiors (96^3 .. 256^3, seeded), 20-cell PML,
  3-6 horizontal layers each, one Ricker source and 128 receivers per model.
* `balance()` — greedy assignment of models to ranks by computed cells.
* `von_karman_random_field()` — seeded von Karman-spectrum perturbation.
* `gaussian_random_field()` — seeded Gaussian-correlated perturbation used
  for the random media; it stands in for the reference's MATLAB generator
  randomMedium/RandomMedia_3_d.m:1-103, which uses another spectrum.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import (DAMP_LOGR, DAMP_REFGPU, QUIRKS_FIXED, QUIRKS_REF, REF_COEF, TXX, VX, VY, VZ)

HALO = 5


@dataclasses.dataclass
class Workload:
    name: str
    cfg: dict                      # sgfd_config fields
    b: np.ndarray                  # float32, (nz, ny, nx)
    lam: np.ndarray
    mu: np.ndarray
    src: tuple
    rec_xyz: np.ndarray            # (n, 3) int32
    rec_comp: np.ndarray           # (n,) int32
    nt: int
    wavelet: np.ndarray            # float32 (nt,)
    wavelet64: np.ndarray          # float64 (nt,) for FP64 oracle runs

    @property
    def shape(self):
        return (self.cfg["nz"], self.cfg["ny"], self.cfg["nx"])

    def computed_cells(self) -> int:
        c = self.cfg
        return (c["nx"] - 2 * HALO) * (c["ny"] - 2 * HALO) * (c["nz"] - 2 * HALO)


def medium_from_velocity(vp, vs, rho):
    """b = 1/rho, mu = rho vs^2, lambda = rho (vp^2 - 2 vs^2), computed in float64, stored float32."""
    vp = np.asarray(vp, dtype=np.float64)
    vs = np.asarray(vs, dtype=np.float64)
    rho = np.asarray(rho, dtype=np.float64)
    mu = rho * vs * vs
    lam = rho * (vp * vp - 2.0 * vs * vs)
    return (1.0 / rho).astype(np.float32), lam.astype(np.float32), mu.astype(np.float32)


def gaussian_random_field(shape, std, corr_cells, seed):
    """Zero-mean field with autocorrelation ~ exp(-r^2/a^2), a = corr_cells, rescaled to `std`.

    White N(0,1) noise from numpy's PCG64(seed), smoothed by a separable
    Gaussian of sigma = a/2 cells (the convolution of two such Gaussians has
    the requested exp(-r^2/a^2) correlation), then normalised to the sample std.
    """
    from scipy.ndimage import gaussian_filter
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal(size=shape, dtype=np.float32)
    f = gaussian_filter(w, sigma=corr_cells / 2.0, mode="wrap", truncate=4.0)
    f = f.astype(np.float64)
    f -= f.mean()
    f *= std / f.std()
    return f


def von_karman_random_field(shape, std, corr_cells, hurst, seed):
    """Zero-mean field with a von Karman spectrum, rescaled to `std`.

    The 3-D von Karman power spectrum with correlation length a (cells) and
    Hurst exponent H is P(k) ~ (1 + k^2 a^2)^-(H + 3/2) (k in radians per
    cell).  White N(0,1) noise from numpy's PCG64(seed) is filtered in the
    Fourier domain by sqrt(P) (periodic boundaries), then normalised to the
    sample std.  H -> 0.5 is the exponential medium, smaller H is rougher.
    The reference generates its media with a MATLAB script
    (randomMedium/RandomMedia_3_d.m) that cannot run here; this is a seeded
    restatement of the same family of spectra.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    w = rng.standard_normal(size=shape)
    spec = np.fft.rfftn(w)
    ks = [2.0 * np.pi * np.fft.fftfreq(n) for n in shape[:-1]] + [2.0 * np.pi * np.fft.rfftfreq(shape[-1])]
    k2 = ks[0][:, None, None] ** 2 + ks[1][None, :, None] ** 2 + ks[2][None, None, :] ** 2
    spec *= (1.0 + k2 * corr_cells * corr_cells) ** (-(hurst + 1.5) / 2.0)
    f = np.fft.irfftn(spec, s=shape, axes=(0, 1, 2))
    f -= f.mean()
    f *= std / f.std()
    return f


def _cfg(n3, pml, dt, d, damping, quirks, **kw):
    nx, ny, nz = n3
    c = dict(nx=nx, ny=ny, nz=nz, pml=pml, dt=dt, dx=d, dy=d, dz=d, coef=list(REF_COEF),
             damping=damping, damping_R=0.001, damping_vconst=2000.0, quirks=quirks)
    c.update(kw)
    return c


def reference_case(nt: int = 1500) -> Workload:
    """The reference driver's run (CON/main.cu:11-56): GRID 300x200x100, pml 10,
    dt 0.5 ms, 10 m cells, rho 2600, lambda = rho*5000^2, mu = lambda/3,
    source at the grid centre, one txx station 10 cells further along each axis."""
    nx, ny, nz, pml = 300, 200, 100, 10
    shape = (nz, ny, nx)
    # main.cu:53-55 evaluates these in double (pow) and stores float.
    b = np.full(shape, np.float32(1.0) / np.float32(2600.0), np.float32)
    lam = np.full(shape, np.float32(2600.0 * 5000.0 ** 2), np.float32)
    mu = np.full(shape, np.float32(2600.0 * 5000.0 ** 2 / 3.0), np.float32)
    from . import ricker_ref
    w = ricker_ref(20.0, 0.0005, nt)
    return Workload("reference_main_300x200x100", _cfg((nx, ny, nz), pml, 0.0005, 10.0, DAMP_REFGPU, QUIRKS_REF),
                    b, lam, mu, (nx // 2, ny // 2, nz // 2),
                    np.array([[nx // 2 + pml, ny // 2 + pml, nz // 2 + pml]], np.int32),
                    np.array([TXX], np.int32), nt, w, w.astype(np.float64))


def _ricker_t0_64(f0, dt, t0, nt):
    t = np.arange(nt, dtype=np.float64) * dt
    a = math.pi * f0 * (t - t0)
    return (1.0 - 2.0 * a * a) * np.exp(-a * a)


def plain_cube(n_interior: int = 100, pml: int = 20, nt: int = 500, dt: float = 0.001, d: float = 10.0,
               quirks: int = QUIRKS_FIXED, damping: int = DAMP_LOGR) -> Workload:
    """Homogeneous vp 3000, vs 1732, rho 2000; explosive Ricker f0 25 Hz, t0 = 1.2/f0,
    at the centre computed cell; 101 receivers recording vx and vz along x on the
    line 5 cells below the top interior face (the last one is the first PML cell)."""
    n = n_interior + 2 * pml + 2 * HALO
    shape = (n, n, n)
    b, lam, mu = medium_from_velocity(np.full(shape, 3000.0), np.full(shape, 1732.0), np.full(shape, 2000.0))
    c0 = HALO + (n - 2 * HALO) // 2
    z = HALO + pml + 5
    xs = HALO + pml + np.arange(101)
    xs = np.minimum(xs, n - HALO - 1)
    xyz = np.array([[x, c0, z] for x in xs for _ in (0, 1)], np.int32)
    comp = np.array([VX, VZ] * len(xs), np.int32)
    f0 = 25.0
    w64 = _ricker_t0_64(f0, dt, 1.2 / f0, nt)
    return Workload(f"plain_{n_interior}^3+pml{pml}", _cfg((n, n, n), pml, dt, d, damping, quirks),
                    b, lam, mu, (c0, c0, c0), xyz, comp, nt, w64.astype(np.float32), w64)


def random_cube(n_interior: int = 344, pml: int = 20, nt: int = 2000, dt: float = 0.001, d: float = 10.0,
                std: float = 0.05, corr_m: float = 50.0, seed: int = 2, nrec_side: int = 64,
                src_computed=(192, 192, 40), quirks: int = QUIRKS_FIXED, damping: int = DAMP_LOGR,
                spectrum: str = "gaussian", hurst: float = 0.3) -> Workload:
    """Background vp 3000, vs 1732, rho 2000 scaled by (1 + delta), delta a seeded
    Gaussian-correlated field (std, correlation length corr_m); Ricker 20 Hz
    explosive source; nrec_side^2 receivers on the first interior z-plane
    recording vx, vy, vz.  spectrum="von_karman" draws delta from a von Karman
    spectrum (Hurst exponent `hurst`) instead of the Gaussian one."""
    n = n_interior + 2 * pml + 2 * HALO
    shape = (n, n, n)
    if spectrum == "gaussian":
        delta = gaussian_random_field(shape, std, corr_m / d, seed)
    elif spectrum == "von_karman":
        delta = von_karman_random_field(shape, std, corr_m / d, hurst, seed)
    else:
        raise ValueError(f"unknown spectrum {spectrum!r}")
    s = 1.0 + delta
    b, lam, mu = medium_from_velocity(3000.0 * s, 1732.0 * s, 2000.0 * s)
    del delta, s
    i0 = HALO + pml
    ks = i0 + (np.arange(nrec_side) * n_interior) // nrec_side
    z = i0
    pts = [(x, y, z) for y in ks for x in ks]
    xyz = np.array([p for p in pts for _ in range(3)], np.int32)
    comp = np.array([VX, VY, VZ] * len(pts), np.int32)
    src = tuple(int(v) + HALO for v in src_computed)
    f0 = 20.0
    w64 = _ricker_t0_64(f0, dt, 1.2 / f0, nt)
    return Workload(f"random_{n_interior}^3+pml{pml}", _cfg((n, n, n), pml, dt, d, damping, quirks),
                    b, lam, mu, src, xyz, comp, nt, w64.astype(np.float32), w64)


def crop_workload(w: Workload, n_grid: int = 138, pml: int = 20, nt: int = 300) -> Workload:
    """The centre n_grid^3 window of w's medium as a model of its own (128^3
    computed cells with pml 20): source at its centre, Ricker 20 Hz
    (t0 = 1.2/f0), 16x16 receivers 5 cells below the top interior face
    recording vz and txx.  A case the FP64 oracle finishes in seconds, for
    the error of a large configuration's arithmetic against exact arithmetic."""
    nz, ny, nx = w.b.shape
    z0, y0, x0 = (nz - n_grid) // 2, (ny - n_grid) // 2, (nx - n_grid) // 2
    sl = (slice(z0, z0 + n_grid), slice(y0, y0 + n_grid), slice(x0, x0 + n_grid))
    b, lam, mu = (np.ascontiguousarray(a[sl]) for a in (w.b, w.lam, w.mu))
    c = n_grid // 2
    i0, span = HALO + pml, n_grid - 2 * (HALO + pml)
    ks = i0 + (np.arange(16) * span) // 16
    pts = [(x, y, i0 + 5) for y in ks for x in ks]
    xyz = np.array([p for p in pts for _ in (0, 1)], np.int32)
    comp = np.array([VZ, TXX] * len(pts), np.int32)
    cfg = {**w.cfg, "nx": n_grid, "ny": n_grid, "nz": n_grid, "pml": pml}
    w64 = _ricker_t0_64(20.0, w.cfg["dt"], 1.2 / 20.0, nt)
    return Workload(f"crop{n_grid - 10}^3 of {w.name}", cfg, b, lam, mu, (c, c, c), xyz, comp, nt,
                    w64.astype(np.float32), w64)


def small_random_case(nx=37, ny=41, nz=45, pml=6, nt=60, seed=7, quirks=QUIRKS_REF, damping=DAMP_REFGPU,
                      std=0.15, dt=0.0005, d=10.0, nrec=24) -> Workload:
    """A small uneven-size heterogeneous case for bit-exact parity tests: strong
    random perturbation (so the reference's index quirks matter), source and
    receivers anywhere in the computed region, including inside the PML."""
    shape = (nz, ny, nx)
    delta = gaussian_random_field(shape, std, 3.0, seed)
    s = 1.0 + delta
    b, lam, mu = medium_from_velocity(3000.0 * s, 1732.0 * s * (1.0 + 0.3 * delta), 2000.0 * s)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    src = (nx // 2 + 1, ny // 2 - 2, nz // 2 + 3)
    xyz = np.stack([rng.integers(HALO, nx - HALO, nrec), rng.integers(HALO, ny - HALO, nrec),
                    rng.integers(HALO, nz - HALO, nrec)], axis=1).astype(np.int32)
    comp = (np.arange(nrec) % 9).astype(np.int32)
    f0 = 25.0
    w64 = _ricker_t0_64(f0, dt, 1.2 / f0, nt)
    return Workload(f"small_{nx}x{ny}x{nz}_pml{pml}", _cfg((nx, ny, nz), pml, dt, d, damping, quirks),
                    b, lam, mu, src, xyz, comp, nt, w64.astype(np.float32), w64)


# Largest layer vp kept stable at dt = 1 ms, dx = 10 m: the Courant number
# vp dt / dx * sqrt(3) * sum|c_i| (sum|c_i| = 1.316689 for the 10th-order
# coefficients) must stay below 1, i.e. vp < 4385 m/s.  The batched
# configuration draws layer vp up to 4500 m/s, which would blow up; draws
# above the cap are clipped to it.
VP_CFL_CAP = 4380.0


@dataclasses.dataclass
class LayeredSpec:
    """One model of the batched configuration, before its arrays are built."""
    index: int
    n_interior: int
    pml: int
    layer_tops: list           # GRID z index where each layer starts (first is 0)
    vp: list                   # per layer, m/s (after the CFL cap)
    src: tuple                 # GRID coordinates
    f0: float
    nt: int
    dt: float
    d: float
    nrec: int

    @property
    def n(self) -> int:
        return self.n_interior + 2 * self.pml + 2 * HALO

    def computed_cells(self) -> int:
        return (self.n - 2 * HALO) ** 3


def batch_specs(n_models: int = 32, seed: int = 3, nt: int = 1000, dt: float = 0.001, d: float = 10.0,
                pml: int = 20, nrec: int = 128, n_range=(96, 256), vp_range=(1800.0, 4500.0),
                vp_cap: float = VP_CFL_CAP) -> list:
    """Seeded specs of the batched configuration: interior edge ~ U{96..256},
    3-6 horizontal layers with vp ~ U(1800, 4500) clipped at vp_cap, one
    Ricker (f0 ~ U(10, 30) Hz, t0 = 1.2/f0) at a random interior cell."""
    rng = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for i in range(n_models):
        ni = int(rng.integers(n_range[0], n_range[1] + 1))
        n = ni + 2 * pml + 2 * HALO
        nl = int(rng.integers(3, 7))
        tops = [0] + sorted(int(t) for t in rng.choice(np.arange(HALO + pml + 1, n - HALO - pml), nl - 1,
                                                        replace=False))
        vp = [float(min(v, vp_cap)) for v in rng.uniform(vp_range[0], vp_range[1], nl)]
        lo, hi = HALO + pml, n - HALO - pml
        src = tuple(int(v) for v in rng.integers(lo, hi, 3))
        f0 = float(rng.uniform(10.0, 30.0))
        specs.append(LayeredSpec(i, ni, pml, tops, vp, src, f0, nt, dt, d, nrec))
    return specs


def layered_model(spec: LayeredSpec, quirks: int = QUIRKS_FIXED, damping: int = DAMP_LOGR) -> Workload:
    """Arrays of one batched model: horizontal layers (vs = vp/sqrt(3),
    rho = 310 vp^0.25, Gardner), receivers on a 16x8 grid of the plane 5 cells
    below the top interior face recording vz."""
    n = spec.n
    vp_z = np.empty(n)
    for k, top in enumerate(spec.layer_tops):
        vp_z[top:] = spec.vp[k]
    vs_z = vp_z / math.sqrt(3.0)
    rho_z = 310.0 * vp_z ** 0.25
    b_z, lam_z, mu_z = medium_from_velocity(vp_z, vs_z, rho_z)
    shape = (n, n, n)
    b, lam, mu = (np.ascontiguousarray(np.broadcast_to(a[:, None, None], shape)) for a in (b_z, lam_z, mu_z))
    i0, span = HALO + spec.pml, spec.n_interior
    nxr = 16
    nyr = max(1, spec.nrec // nxr)
    xs = i0 + (np.arange(nxr) * span) // nxr
    ys = i0 + (np.arange(nyr) * span) // nyr
    z = i0 + 5
    xyz = np.array([(x, y, z) for y in ys for x in xs], np.int32)[:spec.nrec]
    comp = np.full(len(xyz), VZ, np.int32)
    w64 = _ricker_t0_64(spec.f0, spec.dt, 1.2 / spec.f0, spec.nt)
    return Workload(f"layered{spec.index}_{spec.n_interior}^3+pml{spec.pml}",
                    _cfg((n, n, n), spec.pml, spec.dt, spec.d, damping, quirks),
                    b, lam, mu, spec.src, xyz, comp, spec.nt, w64.astype(np.float32), w64)


def balance(cells, nranks: int) -> list:
    """Greedy longest-first assignment of models to ranks: each model, largest
    first, goes to the rank with the fewest cells so far (ties: lowest rank).
    Returns one list of model indices per rank, each in ascending order."""
    load = [0] * nranks
    out = [[] for _ in range(nranks)]
    for i in sorted(range(len(cells)), key=lambda k: (-cells[k], k)):
        r = min(range(nranks), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += cells[i]
    return [sorted(o) for o in out]

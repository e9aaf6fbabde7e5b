"""The learned absorbing strip: training data from the solver's own runs,
training on the GPU, evaluation against the split-field PML.

Training data (`generate`).  For each seeded medium an "extended" model runs
with a wide 40-cell PML around the region of interest; a second, strip-sized
model (pml = 0: it ends at the zero frame) takes, every few steps, the
extended model's state on its window (`Solver.copy_window_from`, on the
device), advances one plain step, and is compared with the extended model's
next state at sampled strip cells (`Solver.sample_fields`).  In the outer
cells of the strip the plain step misses what lies beyond the frame; the
difference, in the MLP's output units, is the target, and the MLP's inputs
are the strip model's state after its step (`Solver.strip_features`).
Optionally (`rollout`, `policy`) the strip model first runs a few steps with
a network's corrections, so that rows also come from the states a learned
strip drifts into.

Training (`train`): minibatch Adam on the GPU (`mlp_train`, hand-written
forward/backward/Adam kernels).

Evaluation (`reflection`): the same interior and source run three ways — a
6-cell learned strip, the same strip without the network, and a 20-cell
split-field PML — and each reports the energy left in the interior once the
direct wave has gone, relative to its peak (what the boundary reflected),
in all and per face.

Gate (`gate`, `boundary`): the PML is the judge and the fallback.  A
calibration run compares, face by face, the energy the learned strip leaves
with the PML's; the strip is used only when no face does worse, otherwise
the model keeps the 20-cell PML.

    python -m sgfd.learned train --out strip_params.npy          (200 runs, seeds 1000-1199)
    python -m sgfd.learned evaluate --params strip_params.npy --steps 1500
    python -m sgfd.learned gate --params strip_params.npy
"""
from __future__ import annotations

import argparse
import math
import os

import numpy as np

from . import (DAMP_LOGR, MLP_PARAMS, QUIRKS_FIXED, ARITH_FAST, Solver, default_config, mlp_train)
from . import workloads as wl

WIDTH = 6          # strip cells per face
EXT_PML = 40       # PML of the extended (ground-truth) runs
PARAMS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "strip_params.npy")
# the same network trained on 200 runs (seeds 1000-1199, 600 strip cells per
# snapshot, 7.3 M rows); it leaves more energy in the interior late in a run
# than the default parameters (12 runs, seeds 1-12, 4000 cells per snapshot)
PARAMS_200_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "strip_params_200runs.npy")
HALO = wl.HALO


def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases, the output layer scaled down so that
    an untrained strip starts close to no correction."""
    rng = np.random.Generator(np.random.PCG64(seed))
    w1 = rng.standard_normal((252, 64)) * math.sqrt(2.0 / 252)
    w2 = rng.standard_normal((64, 64)) * math.sqrt(2.0 / 64)
    w3 = rng.standard_normal((64, 9)) * math.sqrt(2.0 / 64) * 0.01
    p = np.concatenate([w1.ravel(), np.zeros(64), w2.ravel(), np.zeros(64), w3.ravel(), np.zeros(9)])
    assert p.size == MLP_PARAMS
    return p.astype(np.float32)


def load_params(path: str = PARAMS_PATH) -> np.ndarray:
    return np.load(path).astype(np.float32)


def strip_cells(nc: int, w: int = WIDTH) -> np.ndarray:
    """Computed coordinates (x, y, z) of the strip cells of an nc^3 computed region."""
    r = np.arange(nc)
    z, y, x = np.meshgrid(r, r, r, indexing="ij")
    band = lambda a: (a < w) | (a >= nc - w)
    m = band(x) | band(y) | band(z)
    return np.stack([x[m], y[m], z[m]], axis=1).astype(np.int32)


def medium(n_grid: int, seed: int, kind: str):
    """A seeded medium of n_grid^3 GRID cells: 'random' (Gaussian-correlated,
    std 10 %, 40 m) or 'layered' (3-5 horizontal layers, vp 2000-4000 m/s)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (n_grid,) * 3
    if kind == "random":
        d = wl.gaussian_random_field(shape, 0.10, 4.0, seed)
        s = 1.0 + d
        return wl.medium_from_velocity(3000.0 * s, 1732.0 * s, 2000.0 * s)
    nl = int(rng.integers(3, 6))
    tops = np.sort(rng.choice(np.arange(1, n_grid), nl - 1, replace=False))
    vp_l = rng.uniform(2000.0, 4000.0, nl)
    vp = np.empty(n_grid)
    vp[:] = vp_l[0]
    for k, t in enumerate(tops):
        vp[t:] = vp_l[k + 1]
    vp3 = np.broadcast_to(vp[:, None, None], shape)
    return wl.medium_from_velocity(vp3, vp3 / math.sqrt(3.0), 310.0 * vp3 ** 0.25)


def _cfg(n_grid: int, pml: int, dt: float, d: float, device: int):
    return default_config(nx=n_grid, ny=n_grid, nz=n_grid, pml=pml, dt=dt, dx=d, dy=d, dz=d, coef=wl.REF_COEF,
                          damping=DAMP_LOGR, damping_R=0.001, quirks=QUIRKS_FIXED, arith=ARITH_FAST, device=device)


def generate(seeds, n_int: int = 32, nt: int = 220, first: int = 30, every: int = 3, per_snapshot: int = 4000,
             dt: float = 0.001, d: float = 10.0, device: int = 0, progress: bool = False, rollout=(0,),
             policy=None):
    """Training rows (X [n][252], Y [n][9]) from one extended run per seed
    (seeds alternate random and layered media, Ricker f0 ~ U(15, 30) Hz at
    the centre).  With rollout lengths other than 0 and a policy network,
    each snapshot first lets the strip model run r steps (r drawn from
    `rollout`) with that network's corrections next to the wide run, so that
    the rows also cover the states a learned strip drifts into."""
    nd = n_int + 2 * WIDTH + 2 * HALO            # strip model GRID
    ne = nd + 2 * EXT_PML                        # extended model GRID
    win = slice(EXT_PML, EXT_PML + nd)
    cells_all = strip_cells(nd - 2 * HALO)
    Xs, Ys = [], []
    for k, seed in enumerate(seeds):
        rng = np.random.Generator(np.random.PCG64(10_000 + seed))
        b, lam, mu = medium(ne, seed, "random" if k % 2 == 0 else "layered")
        f0 = float(rng.uniform(15.0, 30.0))
        t = np.arange(nt + 1) * dt - 1.2 / f0
        wav = ((1 - 2 * (math.pi * f0 * t) ** 2) * np.exp(-(math.pi * f0 * t) ** 2)).astype(np.float32)
        E = Solver(_cfg(ne, EXT_PML, dt, d, device))
        D = Solver(_cfg(nd, 0, dt, d, device))
        try:
            E.set_medium(b, lam, mu)
            c = ne // 2
            E.set_source(c, c, c)
            D.set_medium(*(np.ascontiguousarray(a[win, win, win]) for a in (b, lam, mu)))
            it = 0
            while it < nt:
                E.step(it, float(wav[it]))
                if it >= first and (it - first) % every == 0 and it + 1 < nt:
                    r = int(rng.choice(rollout)) if policy is not None and len(rollout) > 1 else 0
                    r = min(r, nt - it - 2)
                    # the strip model takes the wide run's state on its window (frame zero)
                    D.copy_window_from(E, EXT_PML, EXT_PML, EXT_PML)
                    if r > 0:                                 # r steps with the policy's corrections
                        D.set_learned_strip(WIDTH, policy)
                        for j in range(1, r + 1):
                            D.step(it + j, 0.0)
                            E.step(it + j, float(wav[it + j]))
                        D.set_learned_strip(0)
                        it += r
                    D.step(it + 1, 0.0)                       # one plain step of the strip model
                    pick = cells_all[rng.choice(len(cells_all), min(per_snapshot, len(cells_all)), replace=False)]
                    tilde = D.sample_fields(pick)
                    E.step(it + 1, float(wav[it + 1]))
                    true = E.sample_fields(pick + EXT_PML)    # the same cells in the wide run
                    X, s, z = D.strip_features(WIDTH, pick)
                    keep = s > 0
                    if keep.any():
                        y = true[keep] - tilde[keep]
                        y[:, :3] *= z[keep, None]
                        y /= s[keep, None]
                        Xs.append(X[keep])
                        Ys.append(y.astype(np.float32))
                    it += 2
                    continue
                it += 1
        finally:
            E.close()
            D.close()
        if progress and (k + 1) % 20 == 0:
            print(f"generated {k + 1} runs, {sum(len(x) for x in Xs)} rows", flush=True)
    return np.concatenate(Xs), np.concatenate(Ys)


def train(X, Y, epochs: int = 30, batch: int = 4096, lr: float = 1e-3, seed: int = 0, device: int = 0):
    """Shuffle the rows once (seeded), then minibatch Adam on the GPU."""
    rng = np.random.Generator(np.random.PCG64(seed))
    perm = rng.permutation(len(X))
    p, hist = mlp_train(init_params(seed), X[perm], Y[perm], epochs, batch, lr, device)
    return p, hist


def energy_density(fields, b, lam, mu, win) -> np.ndarray:
    """Kinetic + strain energy per cell (the sgfd_energy formulas) of a window."""
    v = [fields[k][win].astype(np.float64) for k in range(9)]
    bb, la, m = (a[win].astype(np.float64) for a in (b, lam, mu))
    ek = 0.5 * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2) / bb
    tr = v[3] + v[4] + v[5]
    ss = v[3] ** 2 + v[4] ** 2 + v[5] ** 2 + 2 * (v[6] ** 2 + v[7] ** 2 + v[8] ** 2)
    return ek + (ss - la / (3 * la + 2 * m) * tr * tr) / (4 * m)


def energy(fields, b, lam, mu, win) -> float:
    """Kinetic + strain energy (the sgfd_energy formulas) of a cubic window."""
    v = [fields[k][win].astype(np.float64) for k in range(9)]
    bb, la, m = (a[win].astype(np.float64) for a in (b, lam, mu))
    ek = 0.5 * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2) / bb
    tr = v[3] + v[4] + v[5]
    ss = v[3] ** 2 + v[4] ** 2 + v[5] ** 2 + 2 * (v[6] ** 2 + v[7] ** 2 + v[8] ** 2)
    es = (ss - la / (3 * la + 2 * m) * tr * tr) / (4 * m)
    return float(ek.sum() + es.sum())


FACES = ("x-", "x+", "y-", "y+", "z-", "z+")


def face_masks(n: int) -> np.ndarray:
    """For an n^3 interior, a boolean mask per face (FACES order) of the cells
    nearer to that face than to any other (ties go to the first face): the
    part of the interior whose late energy that face reflected."""
    r = np.arange(n)
    z, y, x = np.meshgrid(r, r, r, indexing="ij")
    dist = np.stack([x, n - 1 - x, y, n - 1 - y, z, n - 1 - z])
    near = np.argmin(dist, axis=0)
    return np.stack([near == k for k in range(6)])


def reflection(params, seed: int = 999, n_int: int = 48, nt: int = 400, sample_every: int = 20,
               dt: float = 0.001, d: float = 10.0, device: int = 0, media=None) -> dict:
    """Energy left in the n_int^3 interior at the end relative to its peak, for
    the learned 6-cell strip, the bare 6-cell strip (no network) and a 20-cell
    split-field PML, on one seeded random medium (or on `media` = (b, lam, mu)
    of (n_int + 50)^3 GRID cells) with a centred Ricker.  Also the final
    energy of each face's part of the interior (face_masks) over the peak."""
    pml20 = 20
    n_big = n_int + 2 * pml20 + 2 * HALO
    if media is None:
        b, lam, mu = medium(n_big, seed, "random")
    else:
        b, lam, mu = (np.asarray(a, np.float32) for a in media)
        assert b.shape == (n_big,) * 3, f"calibration media must be {n_big}^3 GRID cells"
    masks = face_masks(n_int)
    f0 = 20.0
    t = np.arange(nt) * dt - 1.2 / f0
    wav = ((1 - 2 * (math.pi * f0 * t) ** 2) * np.exp(-(math.pi * f0 * t) ** 2)).astype(np.float32)
    out = {}
    for name, width, pml in (("learned_strip", WIDTH, 0), ("bare_strip", WIDTH, 0), ("pml20", pml20, pml20)):
        n = n_int + 2 * width + 2 * HALO
        off = pml20 - width
        cut = slice(off, off + n)
        mb, ml, mm = (np.ascontiguousarray(a[cut, cut, cut]) for a in (b, lam, mu))
        s = Solver(_cfg(n, pml, dt, d, device))
        try:
            s.set_medium(mb, ml, mm)
            s.set_source(n // 2, n // 2, n // 2)
            s.set_wavelet(wav)
            if name == "learned_strip":
                s.set_learned_strip(WIDTH, params)
            inner = slice(HALO + width, HALO + width + n_int)
            hist = []
            for it0 in range(0, nt, sample_every):
                s.run(it0, min(sample_every, nt - it0))
                f = [s.field(k) for k in range(9)]
                hist.append(energy(f, mb, ml, mm, (inner, inner, inner)))
            dens = energy_density(f, mb, ml, mm, (inner, inner, inner))
        finally:
            s.close()
        hist = np.array(hist)
        out[name] = {"final_over_peak": float(hist[-1] / hist.max()), "peak": float(hist.max()),
                     "history": hist.tolist(),
                     "face_final_over_peak": {fc: float(dens[masks[k]].sum() / hist.max())
                                              for k, fc in enumerate(FACES)}}
    return out


def gate(params, nt: int = 400, seed: int = 999, media=None, margin: float = 1.0, device: int = 0) -> dict:
    """The learned strip's gate: the split-field PML is the judge and the
    fallback.  A calibration run (reflection(): the same medium and source
    with the learned 6-cell strip and with a 20-cell PML) measures, per face,
    the energy that face's part of the interior still holds after nt steps.
    A face accepts the strip when its energy is no larger than margin times
    the PML's.  The solver runs one boundary kind on all six faces, so the
    strip is used only if every face accepts it; otherwise the model keeps
    the PML.  Returns the decision ("learned_strip" or "pml20"), the faces'
    verdicts and the measured energies."""
    r = reflection(params, seed=seed, nt=nt, sample_every=max(1, nt // 8), device=device, media=media)
    learned, pml = r["learned_strip"], r["pml20"]
    faces = {fc: bool(np.isfinite(learned["face_final_over_peak"][fc]) and
                      learned["face_final_over_peak"][fc] <= margin * pml["face_final_over_peak"][fc])
             for fc in FACES}
    total_ok = bool(np.isfinite(learned["final_over_peak"]) and
                    learned["final_over_peak"] <= margin * pml["final_over_peak"])
    use = all(faces.values()) and total_ok
    return {"boundary": "learned_strip" if use else "pml20", "faces_accept": faces, "steps": nt,
            "learned_final_over_peak": learned["final_over_peak"], "pml_final_over_peak": pml["final_over_peak"],
            "learned_faces": learned["face_final_over_peak"], "pml_faces": pml["face_final_over_peak"]}


def boundary(params, decision: dict) -> dict:
    """Solver settings for a gate decision: the learned strip (pml = 0 and the
    strip's width and parameters for set_learned_strip) or the 20-cell PML."""
    if decision["boundary"] == "learned_strip":
        return {"pml": 0, "strip_width": WIDTH, "params": params}
    return {"pml": 20, "strip_width": 0, "params": None}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=PARAMS_PATH)
    t.add_argument("--runs", type=int, default=200)
    t.add_argument("--seed0", type=int, default=1000, help="first seed (seeds seed0 .. seed0+runs-1)")
    t.add_argument("--per-snapshot", type=int, default=600, help="strip cells sampled per snapshot")
    t.add_argument("--epochs", type=int, default=30)
    t.add_argument("--nt", type=int, default=220, help="steps of each wide run")
    t.add_argument("--rollout", default="0", help="comma-separated rollout lengths drawn per snapshot")
    t.add_argument("--policy", default=PARAMS_PATH, help="network that runs the rollouts")
    t.add_argument("--device", type=int, default=0)
    g = sub.add_parser("gate")
    g.add_argument("--params", default=PARAMS_PATH)
    g.add_argument("--steps", type=int, default=400)
    g.add_argument("--device", type=int, default=0)
    e = sub.add_parser("evaluate")
    e.add_argument("--params", default=PARAMS_PATH)
    e.add_argument("--steps", type=int, default=400)
    e.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    if a.cmd == "train":
        roll = tuple(int(v) for v in a.rollout.split(","))
        X, Y = generate(range(a.seed0, a.seed0 + a.runs), nt=a.nt, per_snapshot=a.per_snapshot, device=a.device,
                        progress=True, rollout=roll, policy=load_params(a.policy) if max(roll) > 0 else None)
        p, hist = train(X, Y, epochs=a.epochs, device=a.device)
        np.save(a.out, p)
        print({"rows": len(X), "epoch_loss": [round(float(v), 6) for v in hist]}, flush=True)
        for n in (400, 1500):
            r = reflection(p, nt=n, sample_every=50, device=a.device)
            hist_l = r["learned_strip"]["history"]
            print(n, {k: v["final_over_peak"] for k, v in r.items()},
                  "second-half growth", hist_l[-1] / hist_l[len(hist_l) // 2], flush=True)
    elif a.cmd == "gate":
        print(gate(np.load(a.params), nt=a.steps, device=a.device), flush=True)
    else:
        r = reflection(np.load(a.params), nt=a.steps, sample_every=50 if a.steps > 400 else 20, device=a.device)
        print({k: v["final_over_peak"] for k, v in r.items()}, flush=True)


if __name__ == "__main__":
    main()

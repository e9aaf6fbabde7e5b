"""Shared helpers for the tests: run one workload on the oracle or on the GPU."""
import numpy as np

import oracle_py


def run_oracle(w, fp64=False, ftz=False, nsteps=None):
    o = oracle_py.Oracle(w.cfg, fp64=fp64, ftz=ftz)
    o.set_medium(w.b, w.lam, w.mu)
    o.set_source(*w.src)
    o.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
    o.run(w.wavelet64 if fp64 else w.wavelet.astype(np.float64), 0, nsteps if nsteps is not None else w.nt)
    return o


def make_solver(w, **overrides):
    import sgfd
    cfg = sgfd.default_config(**{**w.cfg, **overrides})
    s = sgfd.Solver(cfg)
    s.set_medium(w.b, w.lam, w.mu)
    s.set_source(*w.src)
    s.set_receivers(w.rec_xyz, w.rec_comp, w.nt)
    s.set_wavelet(w.wavelet)
    return s

"""CPU checks of the MLP oracle: its gradient against central finite
differences of its own loss (so that the GPU gradients are checked against
something pinned)."""
import numpy as np

import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.standard_normal(mo.N_PARAMS) * 0.1
    X = rng.standard_normal((7, mo.N_IN))
    Y = rng.standard_normal((7, mo.N_OUT))
    _, g = mo.loss_and_gradient(p, X, Y)
    idx = rng.choice(mo.N_PARAMS, 60, replace=False)
    idx = np.concatenate([idx, [mo.N_PARAMS - 1, 0, 16128, 20288]])   # one from every block
    h = 1e-6
    for i in idx:
        e = np.zeros(mo.N_PARAMS)
        e[i] = h
        fd = (mo.loss_and_gradient(p + e, X, Y)[0] - mo.loss_and_gradient(p - e, X, Y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    assert mo.N_PARAMS == 20937

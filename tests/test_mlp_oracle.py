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


def test_f16_forward_rounds_operands_and_stays_near_fp64():
    """forward_f16 rounds to binary16 with ties to even, and the FP16 operand
    rounding moves the network's outputs by well under 1e-2 of the largest."""
    assert mo.f16(1.0 + 2.0 ** -11) == 1.0                    # tie -> even
    assert mo.f16(1.0 + 3 * 2.0 ** -11) == 1.0 + 2.0 ** -9    # tie -> even (up)
    assert mo.f16(65504.0) == 65504.0 and mo.f16(2.0 ** -24) == 2.0 ** -24
    rng = np.random.default_rng(2)
    p = rng.standard_normal(mo.N_PARAMS) * 0.1
    X = rng.standard_normal((256, mo.N_IN))
    exact, _ = mo.forward(p, X)
    approx = mo.forward_f16(p, X)
    err = np.abs(approx - exact).max() / np.abs(exact).max()
    assert 1e-5 < err < 1e-2, err


def test_face_masks_partition_the_interior():
    """Every interior cell belongs to exactly one face's part, opposite faces'
    parts are mirror images (even edge), and a cell next to a face belongs to it."""
    import sgfd.learned as L
    m = L.face_masks(12)
    assert m.shape == (6, 12, 12, 12)
    np.testing.assert_array_equal(m.sum(axis=0), 1)
    assert m[0, 6, 6, 0] and m[1, 6, 6, 11] and m[2, 6, 0, 6] and m[3, 6, 11, 6] and m[4, 0, 6, 6] and m[5, 11, 6, 6]
    sizes = m.reshape(6, -1).sum(axis=1)
    assert sizes.min() > 0 and sizes[0] == sizes[1] and sizes[2] == sizes[3] and sizes[4] == sizes[5]
    np.testing.assert_array_equal(m[0], m[1][:, :, ::-1])

"""Host-side workload logic (no GPU): the batched configuration's seeded specs,
its CFL cap, and the greedy model-to-rank balance used by multi-GPU replicas."""
import math

import numpy as np

import sgfd
import sgfd.workloads as wl


def test_batch_specs_follow_the_configuration():
    specs = wl.batch_specs()
    assert len(specs) == 32
    assert specs == wl.batch_specs()                       # seeded
    for s in specs:
        assert 96 <= s.n_interior <= 256 and s.pml == 20
        assert 3 <= len(s.vp) <= 6 and len(s.layer_tops) == len(s.vp) and s.layer_tops[0] == 0
        assert all(1800.0 <= v <= wl.VP_CFL_CAP for v in s.vp)
        assert 10.0 <= s.f0 <= 30.0
        lo, hi = wl.HALO + s.pml, s.n - wl.HALO - s.pml
        assert all(lo <= c < hi for c in s.src)
    courant = wl.VP_CFL_CAP * 0.001 / 10.0 * math.sqrt(3.0) * float(np.abs(sgfd.REF_COEF).sum())
    assert courant < 1.0
    total = sum(s.computed_cells() for s in specs)
    assert 3.0e8 < total < 4.2e8


def test_layered_model_arrays():
    spec = wl.batch_specs(n_models=1, n_range=(40, 40), pml=6, nt=50, nrec=32)[0]
    w = wl.layered_model(spec)
    n = spec.n
    assert w.b.shape == (n, n, n) and w.b.dtype == np.float32
    assert len(w.rec_comp) == 32 and (w.rec_comp == sgfd.VZ).all()
    # horizontal layers: constant in x and y, Gardner density, vp/vs = sqrt(3)
    assert (w.mu == w.mu[:, :1, :1]).all()
    rho = 1.0 / w.b[:, 0, 0].astype(np.float64)
    vs = np.sqrt(w.mu[:, 0, 0] / rho)
    vp = np.sqrt((w.lam[:, 0, 0] + 2 * w.mu[:, 0, 0]) / rho)
    np.testing.assert_allclose(vp / vs, math.sqrt(3.0), rtol=1e-5)
    np.testing.assert_allclose(rho, 310.0 * vp ** 0.25, rtol=1e-5)
    assert len(np.unique(w.mu[:, 0, 0])) <= len(spec.vp)


def test_balance_is_a_partition_within_one_model_of_even():
    rng = np.random.default_rng(0)
    for nranks in (1, 2, 3, 4, 8):
        cells = [int(c) for c in rng.integers(1_000, 20_000_000, 32)]
        parts = wl.balance(cells, nranks)
        assert sorted(i for p in parts for i in p) == list(range(32))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)
    assert wl.balance([5, 5], 4) == [[0], [1], [], []]


def test_random_fields_are_seeded_normalised_and_ordered_by_roughness():
    shape = (32, 40, 48)
    g = wl.gaussian_random_field(shape, 0.05, 5.0, 2)
    assert np.array_equal(g, wl.gaussian_random_field(shape, 0.05, 5.0, 2))
    rough = wl.von_karman_random_field(shape, 0.05, 5.0, 0.1, 2)
    smooth = wl.von_karman_random_field(shape, 0.05, 5.0, 1.0, 2)
    for f in (g, rough, smooth):
        assert abs(f.mean()) < 1e-12 and abs(f.std() - 0.05) < 1e-12 and f.shape == shape
    assert np.array_equal(rough, wl.von_karman_random_field(shape, 0.05, 5.0, 0.1, 2))
    grad = lambda f: float(np.mean(np.diff(f, axis=2) ** 2))
    assert grad(rough) > grad(smooth)
    # a longer correlation length gives a smoother field
    assert grad(wl.von_karman_random_field(shape, 0.05, 10.0, 0.5, 3)) < grad(
        wl.von_karman_random_field(shape, 0.05, 2.0, 0.5, 3))
    w = wl.random_cube(n_interior=20, pml=4, nt=10, spectrum="von_karman", nrec_side=4)
    assert w.b.shape == (38, 38, 38)

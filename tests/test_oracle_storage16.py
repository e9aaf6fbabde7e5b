"""CPU checks of the 16-bit storage emulation in the oracle: its roundings
against numpy's (binary16) and a bit-level bfloat16 restatement, and the
per-field scales it chooses."""
import numpy as np

import oracle_py
import sgfd
import sgfd.workloads as wl
from helpers import run_oracle


def _bf16_numpy(x):
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _edge_values():
    rng = np.random.default_rng(5)
    v = np.concatenate([
        rng.standard_normal(20000).astype(np.float32) * np.float32(10.0) ** rng.integers(-9, 6, 20000),
        np.float32([0.0, -0.0, 65504.0, 65519.9, 65520.0, 7e4, -7e4, 6.1035156e-05, 5.96e-08, 2.98e-08,
                    2.99e-08, 1e-9, 3.0e38, -1.17549435e-38, 1.0 + 2.0 ** -11, 1.0 + 3 * 2.0 ** -11]),
    ])
    return v.astype(np.float32)


def test_binary16_rounding_matches_numpy():
    v = _edge_values()
    got = oracle_py.round16(sgfd.STORE_F16, v)
    want = v.astype(np.float16).astype(np.float32)
    np.testing.assert_array_equal(got, want)
    assert np.signbit(got[v == 0]).tolist() == np.signbit(v[v == 0]).tolist()


def test_bfloat16_rounding_matches_bit_restatement():
    v = _edge_values()
    np.testing.assert_array_equal(oracle_py.round16(sgfd.STORE_BF16, v), _bf16_numpy(v))


def test_storage_emulation_stores_16_bit_values_and_rescales():
    w = wl.small_random_case(nt=60)
    w.cfg["storage"] = sgfd.STORE_F16
    o = run_oracle(w)
    e = o.scale_exponents()
    for fid in range(9):
        f = o.field(fid).astype(np.float32)
        h = f * np.float32(2.0) ** -int(e[fid])           # stored values, exactly
        np.testing.assert_array_equal(h, h.astype(np.float16).astype(np.float32))
        m = np.abs(f).max()
        assert m > 0, fid   # every field got a scale that keeps it off zero
        # chosen after step 49 from that step's largest value: the stored
        # maximum sits near 2^7, well inside binary16's range
        assert 2.0 ** 4 <= np.abs(h).max() < 2.0 ** 11, (fid, np.abs(h).max())
    # 16-bit storage stays close to FP32 storage on this short run
    o32 = run_oracle(wl.small_random_case(nt=60))
    err = np.linalg.norm(o.traces() - o32.traces()) / np.linalg.norm(o32.traces())
    assert err < 5e-3, err

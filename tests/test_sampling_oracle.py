"""CPU: the sampling restatement in the oracle (the checker of the GPU shot
sampler) -- its fixed-order scan agrees with a plain running sum to rounding,
its chunk structure is exact at chunk boundaries, and its draws follow the
inverse-CDF rule of rand's WeightedIndex (first running sum above u)."""
import numpy as np

import oracle


def test_scan_matches_running_sum():
    rng = np.random.default_rng(3)
    for N in (1, 5, 1023, 1024, 1025, 4096 + 17, 3 * 1024 * 1024 + 5):
        v = rng.random(N)
        c = oracle._scan(v)
        assert len(c) == N
        assert np.abs(c - np.cumsum(v)).max() <= 1e-12 * max(1.0, float(np.sum(v)))
        assert np.all(np.diff(c) >= 0)


def test_scan_is_exact_on_integers():
    # small integers sum exactly in any order: the scan must equal cumsum
    v = np.arange(1, 5000, dtype=np.float64) % 7
    assert np.array_equal(oracle._scan(v), np.cumsum(v))


def test_inverse_cdf_rule():
    psi = np.sqrt(np.array([0.1, 0.0, 0.2, 0.7])).astype(np.complex128)
    idx = oracle.sample_indices(psi, 200_000, 5)
    assert 1 not in set(idx.tolist())
    freq = np.bincount(idx.astype(np.int64), minlength=4) / len(idx)
    assert np.abs(freq - [0.1, 0.0, 0.2, 0.7]).max() < 5e-3
    # same seed, same shots
    assert np.array_equal(idx, oracle.sample_indices(psi, 200_000, 5))

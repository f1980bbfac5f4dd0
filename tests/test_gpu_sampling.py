"""GPU: shot sampling (State::measure / measure_shots_parallel,
src/states/mod.rs:180-185, 244-258) on the engine's own kernels: |psi_i|^2,
a fixed-order FP64 scan, SplitMix64 uniforms and an inverse-CDF binary search.

The oracle restates every step in numpy (the scan's summation order included),
so the sampled indices must be EQUAL shot for shot -- not just close in
distribution.  The reference draws the same inverse-CDF rule through rand's
WeightedIndex with its own generator; the distribution is checked separately
with a chi-square test."""
import ctypes as C

import numpy as np
import pytest

import oracle
from helpers import random_state
from logosq_b200 import State, abi, workloads
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu


def shots(st, n_shots, seed):
    out = np.empty(n_shots, dtype=np.uint64)
    call("lq_measure_shots", st.handle, C.c_uint64(n_shots), C.c_uint64(seed),
         out.ctypes.data_as(C.POINTER(C.c_uint64)))
    return out


@pytest.mark.parametrize("n,n_shots,seed", [(16, 1_000_000, 7), (22, 1 << 20, 11), (5, 4096, 3),
                                            (11, 100_000, 5)])
def test_shots_equal_oracle_inverse_cdf(n, n_shots, seed):
    # a non-uniform state: brickwork layers on a Gaussian start
    v = random_state(n, 100 + n)
    g = workloads.brickwork_u3(n, 2, seed=9)
    v = oracle.apply_circuit(v.copy(), g)
    st = State.zero_state(n)
    try:
        st.set_vector(v)
        got = shots(st, n_shots, seed)
        got_again = shots(st, n_shots, seed)
    finally:
        st.close()
    want = oracle.sample_indices(v, n_shots, seed)
    assert np.array_equal(got, got_again)
    assert np.array_equal(got, want), int((got != want).sum())


def test_shot_distribution_chi_square():
    from scipy.stats import chi2
    n, n_shots = 8, 2_000_000
    v = oracle.apply_circuit(random_state(n, 41), workloads.brickwork_u3(n, 3, seed=4))
    st = State.zero_state(n)
    try:
        st.set_vector(v)
        got = shots(st, n_shots, 12345)
    finally:
        st.close()
    counts = np.bincount(got.astype(np.int64), minlength=1 << n)
    p = np.abs(v) ** 2
    p = p / p.sum()
    expect = p * n_shots
    keep = expect > 5
    stat = float((((counts - expect) ** 2)[keep] / expect[keep]).sum())
    assert chi2.sf(stat, int(keep.sum()) - 1) > 1e-6, stat


def test_zero_probability_indices_never_drawn():
    n = 12
    v = np.zeros(1 << n, dtype=np.complex128)
    v[[3, 700, 2048, 4095]] = [0.5, 0.5j, -0.5, 0.5]
    st = State.zero_state(n)
    try:
        st.set_vector(v)
        got = shots(st, 200_000, 1)
    finally:
        st.close()
    assert set(np.unique(got).tolist()) == {3, 700, 2048, 4095}
    assert np.array_equal(got, oracle.sample_indices(v, 200_000, 1))


def test_complex64_state_shots_equal_oracle():
    n = 14
    v = oracle.apply_circuit(random_state(n, 8), workloads.brickwork_u3(n, 2, seed=3))
    st = State.zero_state(n, dtype=abi.LQ_C64)
    try:
        st.set_vector(v)
        got = shots(st, 300_000, 99)
    finally:
        st.close()
    v64 = v.astype(np.complex64).astype(np.complex128)  # the state as stored
    assert np.array_equal(got, oracle.sample_indices(v64, 300_000, 99))

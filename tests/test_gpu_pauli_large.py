"""GPU: Pauli-sum expectation of 16- to 22-qubit states (complex128) against the
oracle (PauliObservable::expectation, src/optimization/observable.rs:95-147,
228-232) and against the per-term evaluation (one sweep per term instead of
one per X-mask group), 1e-12 relative: X masks local to a few bits, only in
bits 0-3, at the top bits, across bit 3/4 and spanning the whole index, Z-only
terms, both Y conventions, XYZ chains, and run-to-run determinism."""
import ctypes as C

import numpy as np
import pytest

import oracle
from helpers import random_state
from logosq_b200 import State, abi, workloads
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu
TOL = 1e-12


def expect(st, terms, yc, per_term=False):
    out = C.c_double()
    per = np.zeros(len(terms)) if per_term else None
    call("lq_expectation_pauli", st.handle, abi.term_ptr(terms), len(terms), yc, C.byref(out),
         abi.f64_ptr(per) if per_term else None)
    return out.value, per


def pack(specs):
    terms = np.zeros(len(specs), dtype=abi.TERM_DTYPE)
    for k, (c, x, z) in enumerate(specs):
        terms[k]["coefficient"] = c
        terms[k]["xmask"] = x
        terms[k]["zmask"] = z
        terms[k]["ny"] = bin(x & z).count("1")
    return terms


def local_x_terms(n, count, seed):
    """Random terms whose X bits above bit 3 lie in one random 8-bit range,
    plus Z-only terms and terms with X bits only in bits 0-3."""
    rng = workloads.SplitMix64(seed)
    specs = []
    for t in range(count):
        z = rng.randint(0, (1 << n) - 1)
        kind = t % 4
        if kind == 0:
            x = 0
        elif kind == 1:
            x = rng.randint(1, 15)
        else:
            h = rng.randint(4, n - 8)
            x = (rng.randint(0, 255) << h) | rng.randint(0, 15)
            if x == 0:
                x = 1 << h
        specs.append((rng.uniform(-1, 1), x, z))
    return pack(specs)


def check(n, terms, seed):
    v = random_state(n, seed)
    st = State.zero_state(n)
    try:
        st.set_vector(v)
        for yc in (abi.Y_REFERENCE, abi.Y_TEXTBOOK):
            want = oracle.expectation(v, terms, yc)
            got, _ = expect(st, terms, yc)
            assert abs(got - want) <= TOL * max(1.0, abs(want)), (n, yc, got, want)
            by_term, per = expect(st, terms, yc, per_term=True)
            assert abs(got - by_term) <= TOL * max(1.0, abs(want))
            assert abs(per.sum() - want) <= TOL * max(1.0, abs(want))
    finally:
        st.close()


@pytest.mark.parametrize("n", [16, 18, 20])
def test_random_sums_vs_oracle(n):
    check(n, local_x_terms(n, 48, seed=n), seed=100 + n)


def test_top_bits_and_bit3_straddle():
    n = 17
    top = (1 << (n - 1)) | (1 << (n - 2))
    specs = [(0.7, top, 0), (-0.4, top, top), (0.3, (1 << 3) | (1 << 4), 1 << 4),
             (0.9, (1 << 4) | (1 << 11), 0), (0.2, 0b1111, 0b1010), (1.1, 0, (1 << n) - 1),
             (-0.6, (1 << 5) | (1 << 12) | 1, (1 << 12) | 2)]
    check(n, pack(specs), seed=7)


def test_wide_x_masks():
    n = 18
    specs = [(0.5, (1 << 4) | (1 << 17), 0), (0.25, (1 << 6) | (1 << 7), 1 << 6),
             (-0.8, 0, 0b101)]
    check(n, pack(specs), seed=9)


@pytest.mark.parametrize("n", [16, 20, 22])
def test_xyz_chain_vs_oracle(n):
    coup = workloads.uniform_stream(50 + n, 3 * (n - 1) + 1, -1.0, 1.0)
    terms = workloads.heisenberg_terms(n, coup[:n - 1], coup[n - 1:2 * (n - 1)],
                                       coup[2 * (n - 1):3 * (n - 1)], 0.5 * coup[-1])
    check(n, terms, seed=200 + n)


def test_result_is_deterministic():
    n = 20
    terms = local_x_terms(n, 32, seed=3)
    v = random_state(n, 5)
    st = State.zero_state(n)
    try:
        st.set_vector(v)
        a, _ = expect(st, terms, abi.Y_REFERENCE)
        b, _ = expect(st, terms, abi.Y_REFERENCE)
        assert a == b
    finally:
        st.close()

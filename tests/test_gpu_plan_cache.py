"""GPU: the fused path's plan cache.  A circuit submitted again on the same
handle (same gates, angles and settings) reuses the program already in the
handle's device buffer; anything else that writes that buffer (a Pauli-sum
expectation, a block gate, the precision form) or any change of gates, angles
or fusion width must plan and upload afresh.  Every result is checked against
the oracle at 1e-12."""
import ctypes as C

import numpy as np
import pytest

import oracle
from logosq_b200 import State, abi, workloads
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run(st, n, g, theta=None):
    th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
    call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g),
         None if th is None else abi.f64_ptr(th), 0 if th is None else len(th), abi.EXEC_FUSED)


def test_repeat_and_invalidation():
    n = 14
    g1 = workloads.brickwork_u3(n, 4, seed=21)
    g2 = workloads.brickwork_u3(n, 4, seed=22)
    v = workloads.gaussian_state(n, 3)
    st = State.zero_state(n)
    try:
        want = v.copy()
        st.set_vector(v)
        for g in (g1, g1, g2, g1, g1):  # repeats hit the cache, changes re-plan
            run(st, n, g)
            want = oracle.apply_circuit(want, g)
            assert np.abs(st.vector() - want).max() < TOL
        # another user of the program buffer in between
        terms = workloads.heisenberg_terms(n, [0.4] * (n - 1), [0.2] * (n - 1), [-0.7] * (n - 1),
                                           0.1)
        e = C.c_double()
        call("lq_expectation_pauli", st.handle, abi.term_ptr(terms), len(terms), abi.Y_REFERENCE,
             C.byref(e), None)
        assert abs(e.value - oracle.expectation(want, terms)) < 1e-12 * max(1, abs(e.value))
        run(st, n, g1)
        want = oracle.apply_circuit(want, g1)
        assert np.abs(st.vector() - want).max() < TOL
        # a block gate rewrites the buffer too
        u, _ = np.linalg.qr(np.random.default_rng(1).normal(size=(8, 8)) + 0j)
        m = np.ascontiguousarray(u).view(np.float64).reshape(-1)
        qs = (C.c_int * 3)(13, 8, 6)  # index bits 0, 5, 7
        call("lq_apply_block", st.handle, 3, qs, m.ctypes.data_as(C.POINTER(C.c_double)))
        got_block = st.vector()
        run(st, n, g1)
        want = oracle.apply_circuit(got_block.copy(), g1)
        assert np.abs(st.vector() - want).max() < TOL
    finally:
        st.close()


def test_angles_and_width_are_part_of_the_key():
    n = 12
    tmpl = workloads.basic_entangling_template(n, 2)
    P = 4 * n
    rng = np.random.default_rng(5)
    old = C.c_int()
    call("lq_get_fusion_width", C.byref(old))
    st = State.zero_state(n)
    try:
        for T, seed in ((10, 1), (10, 2), (11, 2), (11, 2), (10, 1)):
            call("lq_set_fusion_width", T)
            th = np.random.default_rng(seed).uniform(-np.pi, np.pi, P)
            call("lq_state_set_basis", st.handle, C.c_uint64(0))
            run(st, n, tmpl, th)
            want = oracle.apply_circuit(oracle.zero_state(n), tmpl, th)
            assert np.abs(st.vector() - want).max() < TOL, (T, seed)
    finally:
        call("lq_set_fusion_width", old.value)
        st.close()

"""CPU: the fused planner and encoder (via lq_plan_dump) against the oracle,
through a numpy emulator of the kernel's addressing and register ops."""
import numpy as np
import pytest

import oracle
import fused_emulator as fe
from helpers import random_state
from logosq_b200 import abi, workloads
from logosq_b200.gates import make_desc

ONE_Q = [abi.H, abi.X, abi.Y, abi.Z, abi.S, abi.T, abi.RX, abi.RY, abi.RZ, abi.PHASE, abi.U3]
TWO_Q = [abi.CNOT, abi.SWAP, abi.CZ, abi.CPHASE, abi.CRX, abi.CRY, abi.CRZ, abi.CPHASE_PARAM,
         abi.RXX, abi.RYY, abi.RZZ]


def random_circuit(n, count, seed):
    rng = workloads.SplitMix64(seed)
    recs = []
    for _ in range(count):
        kind = [*ONE_Q, *TWO_Q, abi.TOFFOLI][rng.randint(0, len(ONE_Q) + len(TWO_Q))]
        k = 3 if kind == abi.TOFFOLI else (2 if kind in TWO_Q else 1)
        qs = []
        while len(qs) < k:
            q = rng.randint(0, n - 1)
            if q not in qs:
                qs.append(q)
        recs.append(make_desc(kind, qs, [rng.uniform(-3, 3) for _ in range(3)]))
    return np.concatenate(recs)


@pytest.mark.parametrize("n,seed", [(7, 1), (9, 2), (13, 3), (14, 14), (15, 5), (16, 6)])
def test_emulated_random_circuits_match_oracle(n, seed):
    g = random_circuit(n, 40 + 3 * n, seed)
    v = random_state(n, seed)
    assert np.abs(fe.run(n, g, v) - oracle.apply_circuit(v.copy(), g)).max() < 1e-12


@pytest.mark.parametrize("n", [7, 12, 16])
def test_emulated_qft_and_brickwork(n):
    v = random_state(n, 1)
    for g in (workloads.qft_gates(n), workloads.brickwork_u3(n, 6, seed=2)):
        assert np.abs(fe.run(n, g, v) - oracle.apply_circuit(v.copy(), g)).max() < 1e-12


def test_plan_uses_few_passes_for_brickwork():
    import ctypes as C
    from logosq_b200._lib import call
    g = workloads.brickwork_u3(30, 20, seed=2)
    p, r, s = C.c_int(), C.c_int(), C.c_int()
    call("lq_plan_circuit", 30, abi.gate_ptr(g), len(g), C.byref(p), C.byref(r), C.byref(s))
    # Pair folding turns each U3 x U3 . CNOT into one 4x4 op whose two bits must
    # share a window, so a 20-layer brickwork needs a few more passes than layers
    # (27 at the default width) but a third of the ops per layer.
    assert s.value == 0 and p.value <= 30


def _two_qubit_layer(n, kind, seed):
    """U3 on every qubit, then `kind` on pairs (0,1), (2,3), ... (both operand
    orders), so every two-qubit gate follows single-qubit gates on both bits."""
    rng = workloads.SplitMix64(seed)
    recs = [make_desc(abi.U3, [q], [rng.uniform(-3, 3) for _ in range(3)]) for q in range(n)]
    for q in range(0, n - 1, 2):
        qs = [q, q + 1] if (q // 2) % 2 == 0 else [q + 1, q]
        recs.append(make_desc(kind, qs, [rng.uniform(-3, 3) for _ in range(3)]))
    return np.concatenate(recs)


@pytest.mark.parametrize("kind", [abi.CNOT, abi.CZ, abi.CPHASE, abi.CRY, abi.SWAP, abi.RXX,
                                  abi.RZZ])
def test_pair_fold_emits_4x4_ops_and_matches_oracle(kind):
    """Single-qubit gates on both bits of a two-qubit gate fold into one 4x4 op
    (encoded with register bits k0 < k1); the emulated program matches the oracle.
    When the two-qubit gate is a permutation times phases (CNOT, CZ, CPhase,
    SWAP, RZZ) the 4x4 is real (F_M2R) and the Euler phases of the single-qubit
    gates go into diagonal tables over the round's register bits (F_DTAB)."""
    n = 10
    g = _two_qubit_layer(n, kind, 3)
    _, _, _, ops, _ = fe.dump(n, g)
    real = kind in (abi.CNOT, abi.CZ, abi.CPHASE, abi.SWAP, abi.RZZ)
    if real:
        # one real pair op (two scaled rotations and the permutation) per pair,
        # the rotations' scales and the Euler phases in diagonal tables
        pr = ops[ops["type"] == fe.F_PAIR]
        assert len(pr) == n // 2
        assert (pr["k0"] < pr["k1"]).all()
        assert (ops["type"] == fe.F_DTAB).any()
        assert not (ops["type"] == fe.F_M2).any()
    else:
        m2 = ops[ops["type"] == fe.F_M2]
        assert len(m2) == n // 2
        assert (m2["k0"] < m2["k1"]).all()
        assert not (ops["type"] == fe.F_DTAB).any()
    v = random_state(n, 4)
    assert np.abs(fe.run(n, g, v) - oracle.apply_circuit(v.copy(), g)).max() < 1e-12


def _with_width(width, fn):
    import ctypes as C
    from logosq_b200._lib import call
    w0 = C.c_int()
    call("lq_get_fusion_width", C.byref(w0))
    call("lq_set_fusion_width", width)
    try:
        return fn()
    finally:
        call("lq_set_fusion_width", w0.value)


@pytest.mark.parametrize("width", [5, 6, 8, 10, 11, 12])
@pytest.mark.parametrize("n,seed", [(9, 21), (13, 22), (16, 23)])
def test_emulated_random_circuits_at_every_width(width, n, seed):
    """The planner and encoder at every tile width the engine accepts (the
    autotuner picks 10, 11 or 12; lq_set_fusion_width allows 5..12), on random
    circuits of every gate kind."""
    g = random_circuit(n, 30 + 2 * n, seed)
    v = random_state(n, seed)

    def check():
        T = fe.dump(n, g)[0]
        assert T == min(width, n)
        assert np.abs(fe.run(n, g, v) - oracle.apply_circuit(v.copy(), g)).max() < 1e-12

    _with_width(width, check)


@pytest.mark.parametrize("width", [10, 11, 12])
def test_emulated_brickwork_at_autotuned_widths(width):
    n = 16
    g = workloads.brickwork_u3(n, 8, seed=5)
    v = random_state(n, 9)
    _with_width(width, lambda: np.testing.assert_allclose(
        fe.run(n, g, v), oracle.apply_circuit(v.copy(), g), rtol=0, atol=1e-12))


from hypothesis import HealthCheck, given, settings, strategies as st  # noqa: E402


@settings(max_examples=300, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(n=st.integers(5, 12), width=st.integers(5, 12), count=st.integers(1, 60),
       seed=st.integers(0, 2**31 - 1))
def test_planner_property_random_circuits(n, width, count, seed):
    """Any circuit of the engine's gate kinds, at any qubit count and accepted
    tile width, is planned and encoded into passes that the kernel emulator runs
    to the oracle's result."""
    g = random_circuit(n, count, seed)
    v = random_state(n, seed % 1000 + 1)
    _with_width(width, lambda: np.testing.assert_allclose(
        fe.run(n, g, v), oracle.apply_circuit(v.copy(), g), rtol=0, atol=1e-12))


PARAM_KINDS = {abi.RX: 1, abi.RY: 1, abi.RZ: 1, abi.PHASE: 1, abi.U3: 3, abi.CRX: 1, abi.CRY: 1,
               abi.CRZ: 1, abi.CPHASE_PARAM: 1, abi.RXX: 1, abi.RYY: 1, abi.RZZ: 1}


def random_bound_circuit(n, count, nparams, seed):
    """Random circuits whose rotation angles are bound to a parameter vector:
    angle = theta[param] * scale + offset, as an Ansatz template is described."""
    rng = workloads.SplitMix64(seed)
    kinds = list(PARAM_KINDS) + [abi.H, abi.CNOT, abi.CZ, abi.SWAP]
    recs = []
    for _ in range(count):
        kind = kinds[rng.randint(0, len(kinds) - 1)]
        k = 1 if kind in (abi.RX, abi.RY, abi.RZ, abi.PHASE, abi.U3, abi.H) else 2
        qs = []
        while len(qs) < k:
            q = rng.randint(0, n - 1)
            if q not in qs:
                qs.append(q)
        na = PARAM_KINDS.get(kind, 0)
        params = [rng.randint(0, nparams - 1) if rng.uniform() < 0.7 else None for _ in range(na)]
        recs.append(make_desc(kind, qs, [rng.uniform(-1, 1) for _ in range(na)],
                              params=params or None,
                              scales=[rng.uniform(-2, 2) for _ in range(na)] or None))
    return np.concatenate(recs)


@settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(n=st.integers(5, 11), width=st.integers(5, 12), count=st.integers(1, 50),
       nparams=st.integers(1, 12), seed=st.integers(0, 2**31 - 1))
def test_planner_property_parameter_bound_circuits(n, width, count, nparams, seed):
    """Parameter-bound gates (the ansatz templates of the VQE paths) are encoded
    with their angles resolved from theta; the emulated passes match the oracle."""
    g = random_bound_circuit(n, count, nparams, seed)
    theta = np.array([workloads.SplitMix64(seed + i).uniform(-3, 3) for i in range(nparams)])
    v = random_state(n, seed % 1000 + 2)
    _with_width(width, lambda: np.testing.assert_allclose(
        fe.run(n, g, v, theta), oracle.apply_circuit(v.copy(), g, theta), rtol=0, atol=1e-12))


def _unitary(rng, d):
    a = np.array([[complex(rng.uniform(-1, 1), rng.uniform(-1, 1)) for _ in range(d)]
                  for _ in range(d)])
    q, r = np.linalg.qr(a)
    return q * (np.diag(r) / np.abs(np.diag(r)))


@settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.too_slow])
@given(n=st.integers(5, 11), width=st.integers(5, 12), count=st.integers(1, 40),
       seed=st.integers(0, 2**31 - 1))
def test_planner_property_matrix_gates(n, width, count, seed):
    """Explicit 2x2 / 4x4 matrices (Circuit::add_single/two_qubit_gate lowered to
    MATRIX1 / MATRIX2), with and without the renormalising flag of the dense
    builders, mixed with gate structs."""
    rng = workloads.SplitMix64(seed)
    recs = []
    for _ in range(count):
        r = rng.uniform()
        flags = abi.FLAG_RENORM if rng.uniform() < 0.3 else 0
        if r < 0.35:
            recs.append(make_desc(abi.MATRIX1, [rng.randint(0, n - 1)], flags=flags,
                                  matrix=_unitary(rng, 2)))
        elif r < 0.7:
            a = rng.randint(0, n - 1)
            b = (a + 1 + rng.randint(0, n - 2)) % n
            recs.append(make_desc(abi.MATRIX2, [a, b], flags=flags, matrix=_unitary(rng, 4)))
        else:
            recs.append(random_circuit(n, 1, rng.randint(0, 2**31)))
    g = np.concatenate(recs)
    v = random_state(n, seed % 1000 + 3)
    _with_width(width, lambda: np.testing.assert_allclose(
        fe.run(n, g, v), oracle.apply_circuit(v.copy(), g), rtol=0, atol=1e-12))

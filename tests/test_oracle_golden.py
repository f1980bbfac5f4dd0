"""CPU: pin the oracle against the reference's own known answers and numpy.

The reference cannot be compiled here (Rust, no toolchain), so the oracle's
parity rests on (1) every known-answer assertion of the reference tests for this
path (tests/golden/known_answers.json, transcribed with file:line citations),
(2) independent numpy matrix products and the numpy FFT, and (3) the gradient
identities the reference tests assert.
"""
import math

import numpy as np
import pytest

import oracle
from helpers import (build, check_case, known_answers, numpy_apply, oracle_run, random_state,
                     terms_from_strings)
from logosq_b200 import abi, workloads
from logosq_b200.gates import make_desc
from logosq_b200.optimization import (HardwareEfficientAnsatz, Pauli, PauliObservable, PauliTerm,
                                      RealAmplitudesAnsatz, EntanglingGate, EntanglingPattern)

KA = known_answers()


@pytest.mark.parametrize("case", KA["circuits"], ids=lambda c: c["name"])
def test_known_answer_circuits(case):
    c = build(case["n"], case["ops"])
    v = oracle_run(c)
    bad = check_case(v, case["checks"], lambda ops: oracle_run(build(case["n"], ops)))
    assert not bad, f"{case['src']}: {bad}"


@pytest.mark.parametrize("case", KA["observables"], ids=lambda c: c["name"])
def test_known_answer_observables(case):
    v = oracle_run(build(case["n"], case["ops"]))
    terms = terms_from_strings(case["n"], case["terms"])
    assert abs(oracle.expectation(v, terms) - case["value"]) < 1e-10, case["src"]


def test_normalize_known_answers():
    for case in KA["states"]:
        v = np.array([complex(*a) for a in case["vector"]])
        w = oracle.normalize(v.copy())
        nrm = math.sqrt(float(np.sum(np.abs(v) ** 2)))
        expected = v / nrm if nrm > 1e-10 else v
        assert np.abs(w - expected).max() < case["tol"], case["src"]


def test_inner_product_known_answers():
    named = {"zero2": np.array([1, 0, 0, 0], complex), "one2": np.array([0, 0, 0, 1], complex),
             "plus2": np.full(4, 0.5, complex),
             "bell": np.array([1 / math.sqrt(2), 0, 0, 1 / math.sqrt(2)], complex)}
    for case in KA["inner_products"]:
        a = named[case["a"]] if isinstance(case["a"], str) else oracle.normalize(
            np.array([complex(*x) for x in case["a"]]))
        b = named[case["b"]] if isinstance(case["b"], str) else oracle.normalize(
            np.array([complex(*x) for x in case["b"]]))
        got = oracle.inner_product(a, b)
        want = np.vdot(a, b) if case["value"] == "manual" else complex(*case["value"])
        assert abs(got - want) < 1e-10, case["src"]


# ---- every gate kind against an independent numpy product -------------------
def _m(kind, angles):
    c = [math.cos(a / 2) for a in angles[:1]]
    s = [math.sin(a / 2) for a in angles[:1]]
    if kind == abi.H:
        return np.array([[1, 1], [1, -1]]) / math.sqrt(2)
    if kind == abi.X:
        return np.array([[0, 1], [1, 0]])
    if kind == abi.Y:  # the reference struct applies -Y
        return -np.array([[0, -1j], [1j, 0]])
    if kind == abi.Z:
        return np.diag([1, -1])
    if kind == abi.S:
        return np.diag([1, 1j])
    if kind == abi.T:
        return np.diag([1, np.exp(1j * math.pi / 4)])
    if kind == abi.RX:
        return np.array([[c[0], -1j * s[0]], [-1j * s[0], c[0]]])
    if kind == abi.RY:
        return np.array([[c[0], -s[0]], [s[0], c[0]]])
    if kind == abi.RZ:
        return np.diag([np.exp(-0.5j * angles[0]), np.exp(0.5j * angles[0])])
    if kind == abi.PHASE:
        return np.diag([1, np.exp(1j * angles[0])])
    if kind == abi.U3:
        th, ph, la = angles
        return np.array([[math.cos(th / 2), -np.exp(1j * la) * math.sin(th / 2)],
                         [np.exp(1j * ph) * math.sin(th / 2),
                          np.exp(1j * (ph + la)) * math.cos(th / 2)]])
    raise KeyError(kind)


def _ctrl(u):
    m = np.eye(4, dtype=complex)
    m[2:, 2:] = u
    return m


TWO_Q = {
    abi.CNOT: lambda a: _ctrl(np.array([[0, 1], [1, 0]])),
    abi.CZ: lambda a: np.diag([1, 1, 1, -1]),
    abi.SWAP: lambda a: np.eye(4)[[0, 2, 1, 3]],
    abi.CPHASE: lambda a: np.diag([1, 1, 1, np.exp(1j * a[0])]),
    abi.CPHASE_PARAM: lambda a: np.diag([1, 1, 1, np.exp(1j * a[0])]),
    abi.CRX: lambda a: _ctrl(_m(abi.RX, a)),
    abi.CRY: lambda a: _ctrl(_m(abi.RY, a)),
    abi.CRZ: lambda a: _ctrl(_m(abi.RZ, a)),
    abi.RZZ: lambda a: np.diag(np.exp(-0.5j * a[0] * np.array([1, -1, -1, 1]))),
}


@pytest.mark.parametrize("threads", [1, 4])
@pytest.mark.parametrize("kind", [abi.H, abi.X, abi.Y, abi.Z, abi.S, abi.T, abi.RX, abi.RY,
                                  abi.RZ, abi.PHASE, abi.U3])
def test_oracle_one_qubit_gates_vs_numpy(kind, threads):
    oracle.set_threads(threads)
    n = 7
    ang = [0.7, 1.9, -2.3]
    for q in range(n):
        v = random_state(n, 11 + q)
        w = v.copy()
        oracle.apply_circuit(w, make_desc(kind, [q], ang))
        ref = numpy_apply(v, n, _m(kind, ang), [q])
        assert np.abs(w - ref).max() < 1e-14
    oracle.set_threads(1)


@pytest.mark.parametrize("kind", list(TWO_Q))
def test_oracle_two_qubit_gates_vs_numpy(kind):
    n = 6
    for (a, b) in [(0, 1), (1, 0), (0, 5), (5, 0), (2, 4), (4, 2)]:
        v = random_state(n, 100 + a * 7 + b)
        w = v.copy()
        oracle.apply_circuit(w, make_desc(kind, [a, b], [0.83]))
        ref = numpy_apply(v, n, TWO_Q[kind]([0.83]), [a, b])
        assert np.abs(w - ref).max() < 1e-14, (kind, a, b)


def test_oracle_toffoli_vs_numpy():
    n = 5
    m = np.eye(8, dtype=complex)
    m[[6, 7]] = m[[7, 6]]
    for (a, b, t) in [(0, 1, 2), (4, 0, 2), (2, 3, 0)]:
        v = random_state(n, a + 10 * b + 100 * t)
        w = v.copy()
        oracle.apply_circuit(w, make_desc(abi.TOFFOLI, [a, b, t]))
        assert np.abs(w - numpy_apply(v, n, m, [a, b, t])).max() < 1e-14


def test_oracle_rxx_ryy_reference_rule():
    """RXX/RYY skip the |01>,|10> block when qubit1 < qubit2
    (src/gates/parameterized.rs:563-577); textbook mode applies exp(-i t PP/2)."""
    n, th = 4, 0.9
    X = np.array([[0, 1], [1, 0]], complex)
    Yp = np.array([[0, -1j], [1j, 0]])
    for kind, P in ((abi.RXX, X), (abi.RYY, Yp)):
        full = math.cos(th / 2) * np.eye(4) - 1j * math.sin(th / 2) * np.kron(P, P)
        quirk = full.copy()
        quirk[1:3, :] = 0
        quirk[:, 1:3] = 0
        quirk[1, 1] = quirk[2, 2] = 1
        for (a, b) in [(0, 2), (2, 0)]:
            v = random_state(n, 5 + a)
            w = v.copy()
            oracle.apply_circuit(w, make_desc(kind, [a, b], [th]))
            want = numpy_apply(v, n, full if a > b else quirk, [a, b])
            assert np.abs(w - want).max() < 1e-14
            w = v.copy()
            oracle.apply_circuit(w, make_desc(kind, [a, b], [th], flags=abi.FLAG_TEXTBOOK))
            assert np.abs(w - numpy_apply(v, n, full, [a, b])).max() < 1e-14


def test_oracle_threaded_mode_bitwise_identical():
    n = 14
    g = workloads.brickwork_u3(n, 3, seed=2)
    oracle.set_threads(1)
    a = oracle.apply_circuit(oracle.zero_state(n), g)
    oracle.set_threads(8)
    b = oracle.apply_circuit(oracle.zero_state(n), g)
    oracle.set_threads(1)
    assert np.array_equal(a, b)


def test_oracle_qft_matches_fft():
    """qft::apply is an inverse FFT scaled by 1/sqrt(N) (src/algorithms/qft.rs:50-71);
    the gate list of create_circuit must equal it."""
    for n in (3, 8, 12):
        v = random_state(n, 1)
        w = oracle.apply_circuit(v.copy(), workloads.qft_gates(n))
        ref = np.fft.ifft(v) * math.sqrt(len(v))
        assert np.abs(w - ref).max() < 1e-13


def test_oracle_pauli_expectation_vs_numpy():
    n = 6
    v = random_state(n, 3)
    P = {"I": np.eye(2), "X": np.array([[0, 1], [1, 0]]), "Y": np.array([[0, -1j], [1j, 0]]),
         "Z": np.diag([1, -1])}
    for s in ["XYZIZX", "YYIIII", "ZZZZZZ", "IXIYIZ", "YIIIII"]:
        M = np.array([[1.0]])
        for ch in s:
            M = np.kron(M, P[ch])
        textbook = np.vdot(v, M @ v).real
        t = terms_from_strings(n, [[0.7, s]])
        ny = s.count("Y")
        assert abs(oracle.expectation(v, t, abi.Y_TEXTBOOK) - 0.7 * textbook) < 1e-13
        # reference convention: a sign flip per Y factor (src/optimization/observable.rs:125-132)
        assert abs(oracle.expectation(v, t, abi.Y_REFERENCE) - 0.7 * textbook * (-1) ** ny) < 1e-13


def test_oracle_heisenberg_energy_matches_pauli_sum():
    n = 8
    v = random_state(n, 4)
    jx, jy, jz, h = 0.3, -0.7, 1.1, 0.25
    terms = workloads.heisenberg_terms(n, [jx] * (n - 1), [jy] * (n - 1), [jz] * (n - 1), h)
    assert abs(oracle.heisenberg_energy(v, jx, jy, jz, h) - oracle.expectation(v, terms)) < 1e-13


# ---- gradients: tests/test_optimization_gradient.rs --------------------------
def _tpl(ansatz):
    return ansatz.template().packed()


def _obs(o):
    return o.packed()


def test_gradient_known_value():
    """-sin(pi/4) for RY + <Z> (tests/test_optimization_gradient.rs:62-88)."""
    a = HardwareEfficientAnsatz(1, 0, EntanglingGate.CNOT, EntanglingPattern.Linear)
    g = oracle.parameter_shift(1, _tpl(a), [math.pi / 4], _obs(PauliObservable.single_z(1, 0)))
    assert abs(g[0] + math.sin(math.pi / 4)) < 1e-6


def test_gradient_at_extremum():
    a = HardwareEfficientAnsatz(1, 1, EntanglingGate.CNOT, EntanglingPattern.Linear)
    g = oracle.parameter_shift(1, _tpl(a), [0.0, 0.0], _obs(PauliObservable.single_z(1, 0)))
    assert np.all(np.abs(g) < 1e-8)  # tests/test_optimization_gradient.rs:38-60


def test_ps_vs_fd():
    a = RealAmplitudesAnsatz(2, 1)
    p = [0.5, 1.0, 1.5, 0.3, 0.8, 0.2]
    o = _obs(PauliObservable.single_z(2, 0))
    ps = oracle.parameter_shift(2, _tpl(a), p, o)
    fd = oracle.finite_difference(2, _tpl(a), p, o, eps=1e-5)
    assert np.abs(ps - fd).max() < 1e-4  # tests/test_optimization_gradient.rs:91-113


def test_gradient_linearity_identity_symmetry():
    a = RealAmplitudesAnsatz(2, 1)
    p = [0.5, 1.0, 1.5, 0.3, 0.8, 0.2]
    g1 = oracle.parameter_shift(2, _tpl(a), p, _obs(PauliObservable.single_z(2, 0)))
    o2 = PauliObservable.from_terms(2, [PauliTerm(2.0, [Pauli.Z, Pauli.I])])
    g2 = oracle.parameter_shift(2, _tpl(a), p, _obs(o2))
    assert np.abs(g2 - 2 * g1).max() < 1e-10  # :213-239
    h = HardwareEfficientAnsatz(2, 1, EntanglingGate.CNOT, EntanglingPattern.Linear)
    oi = PauliObservable.from_terms(2, [PauliTerm(1.0, [Pauli.I, Pauli.I])])
    gi = oracle.parameter_shift(2, _tpl(h), [0.5, 1.0, 1.5, 2.0], _obs(oi))
    assert np.all(np.abs(gi) < 1e-10)  # :242-263
    os_ = PauliObservable.from_terms(2, [PauliTerm(1.0, [Pauli.Z, Pauli.I]),
                                         PauliTerm(1.0, [Pauli.I, Pauli.Z])])
    gs = oracle.parameter_shift(2, _tpl(h), [0.5] * 4, _obs(os_))
    assert abs(gs[0] - gs[1]) < 1e-6  # :266-298


def test_vqe_adam_converges_on_single_z():
    a = HardwareEfficientAnsatz(1, 1, EntanglingGate.CNOT, EntanglingPattern.Linear)
    th, e, hist = oracle.vqe_adam(1, _tpl(a), [0.3, 0.2], _obs(PauliObservable.single_z(1, 0)),
                                  lr=0.1, max_iter=300)
    assert e < -0.99 and len(hist) > 1

"""GPU parity: every kernel path against the CPU oracle on identical seeded inputs.

Tolerance: 1e-12 max-abs per amplitude (the bar the reference parity target
states), 1e-12 relative on energies, 1e-10 on gradients.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from helpers import (build, check_case, gpu_run, known_answers, oracle_run, random_state,
                     terms_from_strings)
from logosq_b200 import (Circuit, LogosQError, State, abi, workloads, HardwareEfficientAnsatz,
                         ParameterShift, FiniteDifference, PauliObservable, RealAmplitudesAnsatz,
                         EntanglingGate, EntanglingPattern, VariationalQuantumCircuit)
from logosq_b200._lib import call
from logosq_b200.gates import make_desc

pytestmark = pytest.mark.gpu
TOL = 1e-12
KA = known_answers()

ONE_Q = [abi.H, abi.X, abi.Y, abi.Z, abi.S, abi.T, abi.RX, abi.RY, abi.RZ, abi.PHASE, abi.U3]
TWO_Q = [abi.CNOT, abi.SWAP, abi.CZ, abi.CPHASE, abi.CRX, abi.CRY, abi.CRZ, abi.CPHASE_PARAM,
         abi.RXX, abi.RYY, abi.RZZ]


@pytest.mark.parametrize("case", KA["circuits"], ids=lambda c: c["name"])
def test_known_answer_circuits_gpu(case):
    c = build(case["n"], case["ops"])
    for mode in (abi.EXEC_FUSED, abi.EXEC_PER_GATE):
        v = gpu_run(c, mode=mode)
        bad = check_case(v, case["checks"], lambda ops: gpu_run(build(case["n"], ops), mode=mode))
        assert not bad, f"{case['src']} mode={mode}: {bad}"
        assert np.abs(v - oracle_run(c)).max() < TOL


@pytest.mark.parametrize("case", KA["observables"], ids=lambda c: c["name"])
def test_known_answer_observables_gpu(case):
    st = State.zero_state(case["n"])
    build(case["n"], case["ops"]).execute(st)
    terms = terms_from_strings(case["n"], case["terms"])
    out = C.c_double()
    call("lq_expectation_pauli", st.handle, abi.term_ptr(terms), len(terms), abi.Y_REFERENCE,
         C.byref(out), None)
    assert abs(out.value - case["value"]) < 1e-10, case["src"]


@pytest.mark.parametrize("n", [5, 9, 13])
@pytest.mark.parametrize("kind", ONE_Q)
def test_one_qubit_gate_every_position(kind, n):
    ang = [0.37, -1.21, 2.9]
    for q in range(n):
        v = random_state(n, 1000 + 37 * q + kind)
        d = make_desc(kind, [q], ang)
        st = State.zero_state(n)
        st.set_vector(v)
        call("lq_apply_gate", st.handle, abi.gate_ptr(d), None, 0)
        got = st.vector()
        want = oracle.apply_circuit(v.copy(), d)
        assert np.abs(got - want).max() < TOL, (kind, n, q)


@pytest.mark.parametrize("kind", TWO_Q)
def test_two_qubit_gate_pairs(kind):
    n = 9
    pairs = [(0, 1), (1, 0), (0, 8), (8, 0), (3, 7), (7, 3), (4, 5), (8, 7)]
    for flags in (0, abi.FLAG_TEXTBOOK):
        for (a, b) in pairs:
            v = random_state(n, 2000 + 17 * a + b + kind)
            d = make_desc(kind, [a, b], [0.913], flags=flags)
            st = State.zero_state(n)
            st.set_vector(v)
            call("lq_apply_gate", st.handle, abi.gate_ptr(d), None, 0)
            want = oracle.apply_circuit(v.copy(), d)
            assert np.abs(st.vector() - want).max() < TOL, (kind, a, b, flags)


def test_toffoli_triples():
    n = 8
    for (a, b, t) in [(0, 1, 2), (7, 0, 3), (2, 6, 7), (5, 4, 0)]:
        v = random_state(n, a + 8 * b + 64 * t)
        d = make_desc(abi.TOFFOLI, [a, b, t])
        st = State.zero_state(n)
        st.set_vector(v)
        call("lq_apply_gate", st.handle, abi.gate_ptr(d), None, 0)
        assert np.abs(st.vector() - oracle.apply_circuit(v.copy(), d)).max() < TOL


@pytest.mark.parametrize("n", [8, 12, 14, 17])
def test_random_mixed_circuit_fused_vs_oracle(n):
    """Every gate kind at random positions, fused planner vs the oracle."""
    rng = workloads.SplitMix64(n)
    recs = []
    for _ in range(60 + 4 * n):
        kind = [*ONE_Q, *TWO_Q, abi.TOFFOLI][rng.randint(0, len(ONE_Q) + len(TWO_Q))]
        k = 3 if kind == abi.TOFFOLI else (2 if kind in TWO_Q else 1)
        qs = []
        while len(qs) < k:
            q = rng.randint(0, n - 1)
            if q not in qs:
                qs.append(q)
        recs.append(make_desc(kind, qs, [rng.uniform(-3, 3) for _ in range(3)]))
    g = np.concatenate(recs)
    v = random_state(n, 77)
    want = oracle.apply_circuit(v.copy(), g)
    for mode in (abi.EXEC_FUSED, abi.EXEC_PER_GATE):
        st = State.zero_state(n)
        st.set_vector(v)
        call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, mode)
        assert np.abs(st.vector() - want).max() < TOL, mode


def test_qft_20_qubits_random_state():
    """Plain drop-in config: 20-qubit QFT gate by gate on a seeded Gaussian state."""
    n = 20
    v = random_state(n, 1)
    g = workloads.qft_gates(n)
    oracle.set_threads(oracle.max_threads())
    want = oracle.apply_circuit(v.copy(), g)
    oracle.set_threads(1)
    assert np.abs(want - np.fft.ifft(v) * math.sqrt(len(v))).max() < 1e-12
    for mode in (abi.EXEC_FUSED, abi.EXEC_PER_GATE):
        st = State.zero_state(n)
        st.set_vector(v)
        call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, mode)
        assert np.abs(st.vector() - want).max() < TOL, mode


@pytest.mark.parametrize("n,layers", [(16, 20), (22, 6)])
def test_brickwork_vs_oracle(n, layers):
    g = workloads.brickwork_u3(n, layers, seed=2)
    oracle.set_threads(oracle.max_threads())
    want = oracle.apply_circuit(oracle.zero_state(n), g)
    oracle.set_threads(1)
    st = State.zero_state(n)
    call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, abi.EXEC_FUSED)
    got = st.vector()
    assert np.abs(got - want).max() < TOL
    fid = abs(np.vdot(want, got)) ** 2
    assert abs(fid - 1.0) < 1e-12


def test_block_gate_vs_numpy():
    from helpers import numpy_apply
    n = 10
    rng = np.random.default_rng(5)
    for qubits in ([1, 4, 9], [9, 8, 0, 2], [0, 1, 2, 3]):
        k = len(qubits)
        a = rng.normal(size=(2 ** k, 2 ** k)) + 1j * rng.normal(size=(2 ** k, 2 ** k))
        u, _ = np.linalg.qr(a)
        v = random_state(n, 9)
        st = State.zero_state(n)
        st.set_vector(v)
        m = np.ascontiguousarray(u).view(np.float64).reshape(-1)
        qs = (C.c_int * k)(*qubits)
        call("lq_apply_block", st.handle, k, qs, m.ctypes.data_as(C.POINTER(C.c_double)))
        assert np.abs(st.vector() - numpy_apply(v, n, u, qubits)).max() < TOL


def test_reductions_vs_oracle():
    n = 15
    v = random_state(n, 21) * 1.7
    st = State.zero_state(n)
    st.set_vector(v)
    assert abs(st.norm_sqr() - oracle.norm_sqr(v)) < 1e-12 * oracle.norm_sqr(v)
    assert np.abs(st.probabilities() - oracle.probabilities(v)).max() < 1e-15
    st.normalize()
    assert np.abs(st.vector() - oracle.normalize(v.copy())).max() < TOL
    w = random_state(n, 22)
    st2 = State.zero_state(n)
    st2.set_vector(w)
    got = st.inner_product(st2)
    want = oracle.inner_product(oracle.normalize(v.copy()), w)
    assert abs(got - want) < 1e-12
    assert st.probability(5) == pytest.approx(abs(st.vector()[5]) ** 2, abs=1e-16)
    assert st.probability(1 << n) == 0.0


def test_pauli_sum_vs_oracle_both_conventions():
    n = 14
    v = random_state(n, 31)
    rng = workloads.SplitMix64(3)
    terms = np.zeros(40, dtype=abi.TERM_DTYPE)
    for t in range(40):
        x = rng.randint(0, (1 << n) - 1) if t % 3 else 0
        z = rng.randint(0, (1 << n) - 1)
        terms[t]["coefficient"] = rng.uniform(-1, 1)
        terms[t]["xmask"] = x
        terms[t]["zmask"] = z
        terms[t]["ny"] = bin(x & z).count("1")
    st = State.zero_state(n)
    st.set_vector(v)
    for yc in (abi.Y_REFERENCE, abi.Y_TEXTBOOK):
        out = C.c_double()
        per = np.zeros(40)
        call("lq_expectation_pauli", st.handle, abi.term_ptr(terms), 40, yc, C.byref(out),
             abi.f64_ptr(per))
        want = oracle.expectation(v, terms, yc)
        assert abs(out.value - want) < 1e-12 * max(1.0, abs(want))
        out2 = C.c_double()
        call("lq_expectation_pauli", st.handle, abi.term_ptr(terms), 40, yc, C.byref(out2), None)
        assert abs(out2.value - want) < 1e-12 * max(1.0, abs(want))
        for t in range(40):
            assert abs(per[t] - oracle.expectation(v, terms[t:t + 1], yc)) < 1e-12


def test_heisenberg_energy_vs_oracle():
    n = 16
    v = random_state(n, 41)
    st = State.zero_state(n)
    st.set_vector(v)
    jx, jy, jz, h = 0.4, -0.9, 0.6, 0.3
    from logosq_b200 import xyz_heisenberg
    e = xyz_heisenberg.calculate_energy_efficient(st, jx, jy, jz, h)
    want = oracle.heisenberg_energy(v, jx, jy, jz, h)
    assert abs(e - want) < 1e-12 * max(1, abs(want))


def test_parameter_shift_vs_oracle():
    n, L = 8, 4
    vqc = VariationalQuantumCircuit(n, L)
    rng = workloads.SplitMix64(9)
    theta = np.array([rng.uniform(-math.pi, math.pi) for _ in range(vqc.num_parameters())])
    jx = [rng.uniform(-1, 1) for _ in range(n - 1)]
    jy = [rng.uniform(-1, 1) for _ in range(n - 1)]
    jz = [rng.uniform(-1, 1) for _ in range(n - 1)]
    terms = workloads.heisenberg_terms(n, jx, jy, jz, 0.2)
    tpl = vqc.template().packed()
    want = oracle.parameter_shift(n, tpl, theta, terms)
    obs = PauliObservable(n)
    obs._packed = terms
    obs.terms = [None] * len(terms)
    got = ParameterShift().compute_gradient(vqc, obs, theta)
    assert np.abs(got - want).max() < 1e-10
    e_want = oracle.ansatz_energy(n, tpl, theta, terms)
    st = State.zero_state(n)
    out = C.c_double()
    call("lq_ansatz_energy", st.handle, abi.gate_ptr(tpl), len(tpl), abi.f64_ptr(theta),
         len(theta), abi.term_ptr(terms), len(terms), abi.Y_REFERENCE, C.byref(out))
    assert abs(out.value - e_want) < 1e-12 * max(1, abs(e_want))
    fd = FiniteDifference(1e-6).compute_gradient(vqc, obs, theta)
    assert np.abs(fd - want).max() < 1e-4


def test_reference_gradient_assertions_gpu():
    a = HardwareEfficientAnsatz(1, 0, EntanglingGate.CNOT, EntanglingPattern.Linear)
    g = ParameterShift().compute_gradient(a, PauliObservable.single_z(1, 0), [math.pi / 4])
    assert abs(g[0] + math.sin(math.pi / 4)) < 1e-6
    r = RealAmplitudesAnsatz(2, 1)
    p = [0.5, 1.0, 1.5, 0.3, 0.8, 0.2]
    ps = ParameterShift().compute_gradient(r, PauliObservable.single_z(2, 0), p)
    fd = FiniteDifference(1e-5).compute_gradient(r, PauliObservable.single_z(2, 0), p)
    assert np.abs(ps - fd).max() < 1e-4


def test_measure_shots_distribution():
    st = State.zero_state(1)
    assert st.measure_shots_parallel(100) == {0: 100}
    st = State.plus_state(4)
    counts = st.measure_shots_parallel(160000, seed=3)
    assert len(counts) == 16
    assert all(abs(c - 10000) < 600 for c in counts.values())


def test_error_codes():
    st = State.zero_state(4)
    d = make_desc(abi.H, [4])
    with pytest.raises(LogosQError) as e:
        call("lq_apply_gate", st.handle, abi.gate_ptr(d), None, 0)
    assert e.value.code == abi.LQ_ERR_QUBIT_INDEX
    c = Circuit(5)
    c.cnot(0, 1)
    with pytest.raises(LogosQError) as e:
        c.execute(st)
    assert e.value.code == abi.LQ_ERR_QUBIT_MISMATCH
    d = make_desc(abi.RY, [0], params=[3])
    with pytest.raises(LogosQError) as e:
        call("lq_apply_circuit", st.handle, 4, abi.gate_ptr(d), 1, abi.f64_ptr(np.zeros(2)), 2, 0)
    assert e.value.code == abi.LQ_ERR_PARAM_COUNT
    call("lq_set_alloc_limit", C.c_uint64(1 << 20))
    try:
        with pytest.raises(LogosQError) as e:
            State(20)
        assert e.value.code == abi.LQ_ERR_OOM
    finally:
        call("lq_set_alloc_limit", C.c_uint64(0))
    with pytest.raises(LogosQError) as e:
        State.new(np.ones(3))
    assert e.value.code == abi.LQ_ERR_STATE_DIMENSION


def test_state_constructors_and_tensor_product():
    assert np.allclose(State.one_state(3).vector(), np.eye(8)[7])
    assert np.allclose(State.plus_state(3).vector(), np.full(8, 1 / math.sqrt(8)))
    a, b = random_state(3, 1), random_state(2, 2)
    sa, sb = State.zero_state(3), State.zero_state(2)
    sa.set_vector(a)
    sb.set_vector(b)
    assert np.abs(sa.tensor_product(sb).vector() - np.kron(a, b)).max() < TOL
    s = State.new([2 + 1j, 1 + 3j, -1 + 2j, 0.5 - 0.5j])
    v = np.array([2 + 1j, 1 + 3j, -1 + 2j, 0.5 - 0.5j])
    assert np.abs(s.vector() - v / np.linalg.norm(v)).max() < 1e-15
    z = State.new(np.zeros(4))
    assert np.abs(z.vector()).max() == 0.0


def test_fused_pass_count_and_launches():
    """The fused planner cuts full-state passes well below one per gate."""
    n = 24
    g = workloads.brickwork_u3(n, 4, seed=2)
    st = State.zero_state(n)
    call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, abi.EXEC_FUSED)
    launches, passes = C.c_int(), C.c_int()
    call("lq_last_circuit_stats", st.handle, C.byref(launches), C.byref(passes))
    assert passes.value > 0 and launches.value < len(g) / 4

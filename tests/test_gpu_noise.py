"""GPU: the noise models against the numpy oracle of src/noise/mod.rs (max-abs
1e-12 per amplitude), a noisy circuit (every gate followed by the noise models)
against the oracle run gate by gate with the same seeded draws, and the error
codes."""
import numpy as np
import pytest

import oracle
from helpers import random_state
from logosq_b200 import Circuit, LogosQError, State, abi, noise

pytestmark = pytest.mark.gpu


def on_device(n, v, fn):
    st = State.zero_state(n)
    st.set_vector(v)
    fn(st)
    out = st.vector()
    st.close()
    return out


@pytest.mark.parametrize("n", [5, 12])
def test_pauli_errors_match_oracle(n):
    v = random_state(n, n)
    for q in (0, n // 2, n - 1):
        for kind in (1, 2, 3):
            from logosq_b200._lib import call
            got = on_device(n, v, lambda st: call("lq_noise_pauli", st.handle, q, kind))
            assert np.abs(got - oracle.noise_pauli(v, q, kind)).max() < 1e-12


@pytest.mark.parametrize("n,targets", [(6, [2]), (6, [0, 3, 5]), (13, None), (13, [12, 0, 12])])
def test_amplitude_damping_matches_oracle(n, targets):
    v = random_state(n, 7)
    m = noise.AmplitudeDampingNoise(0.3)
    if targets is not None:
        m = m.with_target_qubits(targets)
    got = on_device(n, v, m.apply)
    want = oracle.noise_amplitude_damping(v, 0.3, range(n) if targets is None else targets)
    assert np.abs(got - want).max() < 1e-12


@pytest.mark.parametrize("targets", [[1], [4, 0, 2], None])
def test_phase_damping_matches_oracle(targets):
    n = 9
    v = random_state(n, 3)
    m = noise.PhaseDampingNoise(0.6)
    if targets is not None:
        m = m.with_target_qubits(targets)
    got = on_device(n, v, m.apply)
    want = oracle.noise_phase_damping(v, 0.6, range(n) if targets is None else targets)
    assert np.abs(got - want).max() < 1e-12


def test_thermal_relaxation_matches_oracle():
    n = 8
    v = random_state(n, 5)
    m = noise.ThermalRelaxationNoise(t1=20.0, t2=25.0, gate_time=2.0).with_target_qubits([1, 6])
    got = on_device(n, v, m.apply)
    pa, pp = m.probabilities()
    want = oracle.noise_phase_damping(oracle.noise_amplitude_damping(v, pa, [1, 6]), pp, [1, 6])
    assert np.abs(got - want).max() < 1e-12


def test_noisy_circuit_matches_oracle_gate_by_gate():
    n = 8
    c = Circuit(n)
    for q in range(n):
        c.u3(q, 0.3 + q, 0.2, -0.4)
    for q in range(n - 1):
        c.cnot(q, q + 1)
    c.rz(3, 0.7)
    dep = noise.DepolarizingNoise(0.3, seed=11)
    amp = noise.AmplitudeDampingNoise(0.05).with_target_qubits([0, 5])
    c.add_noise(dep).add_noise(amp)
    st = State.zero_state(n)
    c.execute(st)
    got = st.vector()
    # oracle: same gates one at a time, same seeded draws in the same order
    ref_dep = noise.DepolarizingNoise(0.3, seed=11)
    psi = oracle.zero_state(n)
    for op in c.operations():
        oracle.apply_circuit(psi, op.desc)
        for q, kind in ref_dep.draw(n):
            psi = oracle.noise_pauli(psi, q, kind)
        psi = np.ascontiguousarray(oracle.noise_amplitude_damping(psi, 0.05, [0, 5]))
    assert np.abs(got - psi).max() < 1e-12
    st.close()


def test_noise_error_codes():
    from logosq_b200._lib import call
    st = State.zero_state(4)
    with pytest.raises(LogosQError) as e:
        call("lq_noise_pauli", st.handle, 4, 1)
    assert e.value.code == abi.LQ_ERR_QUBIT_INDEX
    with pytest.raises(LogosQError) as e:
        noise.AmplitudeDampingNoise(1.5).apply(st)
    assert e.value.code == abi.LQ_ERR_INVALID_ARG
    st.close()
    s64 = State.zero_state(4, dtype=abi.LQ_C64)
    with pytest.raises(LogosQError) as e:
        noise.PhaseDampingNoise(0.1).apply(s64)
    assert e.value.code == abi.LQ_ERR_UNSUPPORTED
    s64.close()

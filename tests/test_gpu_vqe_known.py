"""GPU: the reference's VQE and observable tests (tests/test_optimization.rs:
155-418) through the engine: VQE on single-qubit Z, a two-qubit field, the ZZ
Ising term and with two ansatz families, energy decreasing over a run, the
ansatz/state size check, a zero-depth ansatz, an observable with a
coefficient, the gradient's wall time and run-to-run reproducibility, with the
reference's thresholds."""
import math
import time

import numpy as np
import pytest

from logosq_b200 import (Adam, EntanglingGate, EntanglingPattern, GradientDescent,
                         HardwareEfficientAnsatz, LogosQError, ParameterShift, Pauli,
                         PauliObservable, PauliTerm, RealAmplitudesAnsatz, State, VQE)

pytestmark = pytest.mark.gpu


def hea(n, depth):
    return HardwareEfficientAnsatz(n, depth, EntanglingGate.CNOT, EntanglingPattern.Linear)


def test_vqe_single_qubit_z():
    """tests/test_optimization.rs:155-177"""
    vqe = VQE(hea(1, 1), PauliObservable.single_z(1, 0), ParameterShift(),
              GradientDescent(0.1, 100))
    r = vqe.run([0.1, 0.1])
    assert abs(r.ground_state_energy + 1.0) < 0.1


def test_vqe_two_qubit_hamiltonian():
    """tests/test_optimization.rs:179-204"""
    h = PauliObservable(2)
    h.add_term(PauliTerm(1.0, [Pauli.Z, Pauli.I]))
    h.add_term(PauliTerm(1.0, [Pauli.I, Pauli.Z]))
    r = VQE(hea(2, 2), h, ParameterShift(), Adam(0.1, 100)).run([0.1] * 6)
    assert r.ground_state_energy < 0.0


def test_vqe_ising_model():
    """tests/test_optimization.rs:206-227 (random start, seeded here)"""
    r = VQE(RealAmplitudesAnsatz(2, 2), PauliObservable.zz_interaction(2, 0, 1, -1.0),
            ParameterShift(), Adam(0.1, 50)).run_random()
    assert r.ground_state_energy < 0.5


def test_vqe_energy_decreases():
    """tests/test_optimization.rs:229-251"""
    r = VQE(hea(1, 1), PauliObservable.single_z(1, 0), ParameterShift(),
            GradientDescent(0.1, 50)).run([0.5, 0.5])
    assert r.convergence_history[-1] < r.convergence_history[0]


def test_vqe_with_different_ansatz():
    """tests/test_optimization.rs:253-286"""
    h = PauliObservable.single_z(2, 0)
    r_he = VQE(hea(2, 1), h, ParameterShift(), GradientDescent(0.1, 50)).run_random()
    r_ra = VQE(RealAmplitudesAnsatz(2, 1), h, ParameterShift(),
               GradientDescent(0.1, 50)).run_random()
    assert r_he.ground_state_energy < 1.5 and r_ra.ground_state_energy < 1.5


def test_ansatz_wrong_state_size():
    """tests/test_optimization.rs:294-303"""
    with pytest.raises(LogosQError, match="State qubit count must match ansatz"):
        hea(2, 1).apply(State.zero_state(3), [0.1] * 4)


def test_zero_depth_ansatz_execute():
    """tests/test_optimization.rs:305-321"""
    a = hea(2, 0)
    st = State.zero_state(2)
    a.build_circuit([0.0, 0.0]).execute(st)
    assert abs(st.probability(0) - 1.0) < 1e-10


def test_single_qubit_ansatz_apply():
    """tests/test_optimization.rs:323-333"""
    st = State.zero_state(1)
    RealAmplitudesAnsatz(1, 1).apply(st, [math.pi / 2.0, 0.0])
    assert abs(np.sum(np.abs(st.vector()) ** 2) - 1.0) < 1e-10


def test_observable_with_coefficient():
    """tests/test_optimization.rs:335-349"""
    obs = PauliObservable(1)
    obs.add_term(PauliTerm(2.0, [Pauli.Z]))
    assert abs(obs.expectation(State.zero_state(1)) - 2.0) < 1e-10


def test_gradient_computation_time():
    """tests/test_optimization.rs:369-388"""
    a = hea(3, 2)
    params = [0.1] * a.num_parameters()
    ParameterShift().compute_gradient(a, PauliObservable.single_z(3, 0), params)  # warm
    t0 = time.perf_counter()
    ParameterShift().compute_gradient(a, PauliObservable.single_z(3, 0), params)
    assert time.perf_counter() - t0 < 1.0


def test_vqe_reproducibility():
    """tests/test_optimization.rs:390-417 (RealAmplitudes at depth 1 on two qubits
    has the reference's extra initial layer: 6 parameters)"""
    a, h = RealAmplitudesAnsatz(2, 1), PauliObservable.single_z(2, 0)
    assert a.num_parameters() == 6
    r1 = VQE(a, h, ParameterShift(), GradientDescent(0.1, 30)).run([0.5] * 6)
    r2 = VQE(a, h, ParameterShift(), GradientDescent(0.1, 30)).run([0.5] * 6)
    assert abs(r1.ground_state_energy - r2.ground_state_energy) < 1e-6

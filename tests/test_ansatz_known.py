"""CPU: the structural known answers of the reference's ansatz tests
(tests/test_optimization_ansatz.rs) through the Python mirror: parameter
counts, circuit sizes, the operation count of the full entangling pattern and
the parameter-count error.  Circuit building is host-side (gate descriptors),
so no GPU is needed."""
import pytest

from logosq_b200 import (Circuit, EfficientSU2Ansatz, EntanglingGate, EntanglingPattern,
                         HardwareEfficientAnsatz, LogosQError, ParameterizedCircuit,
                         RealAmplitudesAnsatz, abi)


def test_hardware_efficient_creation():
    """tests/test_optimization_ansatz.rs:13-21"""
    a = HardwareEfficientAnsatz(3, 2, EntanglingGate.CNOT, EntanglingPattern.Linear)
    assert a.num_qubits() == 3
    assert a.num_parameters() == 9  # 3 qubits x (2 layers + 1 final)
    assert a.depth == 2


def test_hardware_efficient_linear_pattern():
    """tests/test_optimization_ansatz.rs:23-34"""
    a = HardwareEfficientAnsatz(4, 1, EntanglingGate.CNOT, EntanglingPattern.Linear)
    c = a.build_circuit([0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8])
    assert c.num_qubits() == 4
    assert len(c.operations()) == 11  # 4 RY + 3 CNOT + 4 RY (the reference's comment)


def test_hardware_efficient_circular_pattern():
    """tests/test_optimization_ansatz.rs:36-42"""
    a = HardwareEfficientAnsatz(3, 1, EntanglingGate.CNOT, EntanglingPattern.Circular)
    assert a.num_parameters() == 6


def test_hardware_efficient_full_pattern():
    """tests/test_optimization_ansatz.rs:44-54"""
    a = HardwareEfficientAnsatz(3, 1, EntanglingGate.CNOT, EntanglingPattern.Full)
    assert len(a.build_circuit([0.1] * 6).operations()) == 9


def test_real_amplitudes():
    """tests/test_optimization_ansatz.rs:71-81"""
    a = RealAmplitudesAnsatz(3, 2)
    assert a.num_qubits() == 3 and a.num_parameters() == 9
    assert a.build_circuit([0.1] * 9).num_qubits() == 3


def test_efficient_su2():
    """tests/test_optimization_ansatz.rs:83-95"""
    a = EfficientSU2Ansatz(2, 1)
    assert a.num_qubits() == 2 and a.num_parameters() == 6


def test_parameterized_circuit_custom():
    """tests/test_optimization_ansatz.rs:97-115"""
    def builder(p):
        c = Circuit(2)
        c.ry(0, p[0])
        c.ry(1, p[1])
        c.cnot(0, 1)
        c.ry(0, p[2])
        return c

    a = ParameterizedCircuit(2, 3, builder)
    assert a.num_parameters() == 3
    assert a.build_circuit([0.5, 1.0, 1.5]).num_qubits() == 2


def test_wrong_parameter_count():
    """tests/test_optimization_ansatz.rs:117-123: the reference panics with
    "Parameter count mismatch"; the mirror raises the matching error."""
    a = HardwareEfficientAnsatz(2, 1, EntanglingGate.CNOT, EntanglingPattern.Linear)
    with pytest.raises(LogosQError, match="Parameter count mismatch") as ei:
        a.build_circuit([0.1, 0.2])
    assert ei.value.code == abi.LQ_ERR_PARAM_COUNT


def test_observable_wrong_qubit_index():
    """tests/test_optimization.rs:288-292: single_z on a qubit the system lacks."""
    from logosq_b200 import PauliObservable
    with pytest.raises(LogosQError, match="Qubit index out of bounds") as ei:
        PauliObservable.single_z(2, 3)
    assert ei.value.code == abi.LQ_ERR_QUBIT_INDEX


def test_zero_depth_and_single_qubit_parameter_counts():
    """tests/test_optimization.rs:305-334 (parameter counts)."""
    assert HardwareEfficientAnsatz(2, 0, EntanglingGate.CNOT,
                                   EntanglingPattern.Linear).num_parameters() == 2
    assert RealAmplitudesAnsatz(1, 1).num_parameters() == 2


def test_ansatz_scaling():
    """tests/test_optimization.rs:351-367"""
    for n in range(1, 5):
        a = HardwareEfficientAnsatz(n, 1, EntanglingGate.CNOT, EntanglingPattern.Linear)
        assert a.build_circuit([0.1] * a.num_parameters()).num_qubits() == n


def test_qft_circuit_creation():
    """tests/test_qft.rs:12-28 and 30-42: names and non-empty operation lists."""
    from logosq_b200 import qft
    c = qft.create_circuit(3)
    assert c.num_qubits() == 3 and "Quantum Fourier Transform" in c.name()
    assert len(c.operations()) > 0
    ci = qft.create_inverse_circuit(3)
    assert ci.num_qubits() == 3 and "Inverse" in ci.name() and len(ci.operations()) > 0

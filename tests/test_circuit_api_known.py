"""CPU: the host-side known answers of the reference's dense circuit tests
(tests/test_circuits_dense.rs:20-211) through the mirror's Circuit: creation
and naming, add_operation with a gates::matrix gate, the qubit-index error,
builder counts, composition, reversal names, clone independence and the Debug
printout."""
import pytest

from logosq_b200 import Circuit, LogosQError, abi
from logosq_b200.gates import x_gate


def test_circuit_creation():
    """tests/test_circuits_dense.rs:20-31"""
    c = Circuit(2)
    assert c.num_qubits() == 2 and len(c.operations()) == 0 and c.name() is None
    n = Circuit(3).with_name("Test Circuit")
    assert n.num_qubits() == 3 and n.name() == "Test Circuit"


def test_adding_operations():
    """tests/test_circuits_dense.rs:33-50"""
    c = Circuit(2)
    c.add_operation(x_gate(), [0], "X on 0")
    assert len(c.operations()) == 1
    assert c.operations()[0].qubits() == [0] and c.operations()[0].name() == "X on 0"
    c.add_operation(x_gate(), [1], "X on 1")
    assert len(c.operations()) == 2
    assert c.operations()[1].qubits() == [1] and c.operations()[1].name() == "X on 1"


def test_invalid_qubit_index():
    """tests/test_circuits_dense.rs:52-61"""
    with pytest.raises(LogosQError, match=r"Invalid qubit index: 2 \(must be < 2\)") as ei:
        Circuit(2).add_operation(x_gate(), [2], "X on 2")
    assert ei.value.code == abi.LQ_ERR_QUBIT_INDEX


def test_composition_length():
    """tests/test_circuits_dense.rs:80-104 (operation count)"""
    a, b = Circuit(2), Circuit(2)
    a.x(0)
    b.h(1)
    a.compose(b)
    assert len(a.operations()) == 2


def test_reversal_names():
    """tests/test_circuits_dense.rs:106-133 (names)"""
    c = Circuit(1)
    c.x(0).h(0)
    r = c.reversed()
    assert len(r.operations()) == 2
    assert r.operations()[0].name() == "reversed_H" and r.operations()[1].name() == "reversed_X"


def test_clone_is_independent():
    """tests/test_circuits_dense.rs:135-153"""
    o = Circuit(2)
    o.h(0).cnot(0, 1)
    k = o.clone()
    assert o.num_qubits() == k.num_qubits() and len(o.operations()) == len(k.operations())
    assert o.name() == k.name()
    o.x(0)
    assert len(o.operations()) == 3 and len(k.operations()) == 2


def test_debug_format():
    """tests/test_circuits_dense.rs:155-170"""
    c = Circuit(1).with_name("Test Circuit")
    c.x(0).h(0)
    s = repr(c)
    assert "Test Circuit" in s and "(1 qubits)" in s and "0: X" in s and "1: H" in s


def test_builder_counts():
    """tests/test_circuits_dense.rs:175-208"""
    import math
    c = Circuit(1)
    c.x(0)
    c.y(0)
    c.z(0)
    c.h(0)
    c.s(0)
    c.t(0)
    c.rx(0, math.pi / 2)
    c.ry(0, math.pi / 2)
    c.rz(0, math.pi / 2)
    assert len(c.operations()) == 9
    c2 = Circuit(2)
    c2.cnot(0, 1)
    c2.swap(0, 1)
    c2.cz(0, 1)
    assert len(c2.operations()) == 3


def test_execute_and_measure_with_noise_delegates(monkeypatch):
    """execute_and_measure_with_noise takes execute_and_measure's steps (as in
    src/circuits/mod.rs:376-411), with the seed passed through."""
    seen = []
    monkeypatch.setattr(Circuit, "execute_and_measure", lambda self, seed=0: seen.append(seed) or [1])
    assert Circuit(1).execute_and_measure_with_noise(seed=7) == [1] and seen == [7]

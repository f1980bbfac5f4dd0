"""GPU: the known answers of the reference's state tests (tests/test_states.rs)
through the engine's State: constructors, normalisation by State::new,
measurement, qubit measurement with collapse, probabilities, tensor products,
a MatrixGate application and the printout.  Tolerance 1e-10, as the reference
asserts."""
import numpy as np
import pytest

from logosq_b200 import State
from logosq_b200.gates import MatrixGate

pytestmark = pytest.mark.gpu
TOL = 1e-10
R2 = 1.0 / np.sqrt(2.0)


def test_creation_and_normalisation():
    """tests/test_states.rs:9-45"""
    s = State.new([2.0, 0.0], 1)
    assert abs(abs(s.vector()[0]) ** 2 - 1.0) < TOL and s.num_qubits() == 1
    assert State.new([1.0, 1.0, 1.0, 1.0]).num_qubits() == 2
    s3 = State.new([1.0] + [0.0] * 7, 3)
    assert abs(abs(s3.vector()[0]) ** 2 - 1.0) < TOL and s3.num_qubits() == 3


def test_zero_one_plus_and_bell_states():
    """tests/test_states.rs:47-95"""
    z = State.zero_state(2).vector()
    assert len(z) == 4 and abs(z[0] - 1.0) < TOL and np.abs(z[1:]).max() < TOL
    o = State.one_state(2).vector()
    assert abs(o[3] - 1.0) < TOL and np.abs(o[:3]).max() < TOL
    p = State.plus_state(2).vector()
    assert np.abs(p - 0.5).max() < TOL
    b = State.bell_state().vector()
    assert np.abs(b - np.array([R2, 0, 0, R2])).max() < TOL


def test_deterministic_measurement():
    """tests/test_states.rs:97-106"""
    assert State.zero_state(1).measure() == 0
    assert State.one_state(1).measure() == 1


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_measure_qubit_collapses(seed):
    """tests/test_states.rs:108-132"""
    assert State.zero_state(1).measure_qubit(0, seed) == 0
    assert State.one_state(1).measure_qubit(0, seed) == 1
    s = State.plus_state(1)
    r = s.measure_qubit(0, seed)
    assert r in (0, 1)
    v = s.vector()
    want = np.array([1.0, 0.0]) if r == 0 else np.array([0.0, 1.0])
    assert np.abs(v - want).max() < TOL


def test_probability():
    """tests/test_states.rs:134-153"""
    z = State.zero_state(1)
    assert abs(z.probability(0) - 1.0) < TOL and abs(z.probability(1)) < TOL
    p = State.plus_state(1)
    assert abs(p.probability(0) - 0.5) < TOL and abs(p.probability(1) - 0.5) < TOL
    b = State.bell_state()
    assert abs(b.probability(0) - 0.5) < TOL and abs(b.probability(3) - 0.5) < TOL
    assert abs(b.probability(1)) < TOL and abs(b.probability(2)) < TOL


def test_tensor_product():
    """tests/test_states.rs:155-178"""
    s00 = State.zero_state(1).tensor_product(State.zero_state(1))
    v = s00.vector()
    assert s00.num_qubits() == 2 and abs(v[0] - 1.0) < TOL and np.abs(v[1:]).max() < TOL
    s01 = State.zero_state(1).tensor_product(State.one_state(1))
    v = s01.vector()
    assert s01.num_qubits() == 2 and abs(v[1] - 1.0) < TOL
    assert max(abs(v[0]), abs(v[2]), abs(v[3])) < TOL


def test_matrix_gate_application():
    """tests/test_states.rs:180-207"""
    x = MatrixGate(np.array([[0, 1], [1, 0]], dtype=np.complex128))
    s = State.zero_state(1)
    s.apply_gate(x)
    assert np.abs(s.vector() - np.array([0.0, 1.0])).max() < TOL
    s = State.one_state(1)
    s.apply_gate(x)
    assert np.abs(s.vector() - np.array([1.0, 0.0])).max() < TOL


def test_print():
    """tests/test_states.rs:209-227"""
    out = State.plus_state(1).print()
    assert "State: 1 qubit" in out
    assert "|0⟩ : 0.7071+0.0000i (p=0.5000)" in out
    assert "|1⟩ : 0.7071+0.0000i (p=0.5000)" in out
    out = State.bell_state().print()
    assert "State: 2 qubits" in out
    assert "|00⟩ : 0.7071+0.0000i (p=0.5000)" in out
    assert "|11⟩ : 0.7071+0.0000i (p=0.5000)" in out


def test_measure_shots_parallel():
    """tests/test_parallel.rs:144-217"""
    assert State.zero_state(1).measure_shots_parallel(100) == {0: 100}
    assert State.one_state(1).measure_shots_parallel(100) == {1: 100}
    plus = State.plus_state(1).measure_shots_parallel(1000, seed=1)
    assert set(plus) <= {0, 1} and 0.3 < plus.get(0, 0) / 1000 < 0.7
    bell = State.bell_state().measure_shots_parallel(200, seed=2)
    assert bell.get(1, 0) == 0 and bell.get(2, 0) == 0
    c0, c3 = bell.get(0, 0), bell.get(3, 0)
    assert c0 > 0 and c3 > 0 and 0.3 < c0 / (c0 + c3) < 0.7


def test_normalize_keeps_normalised_state():
    """tests/test_parallel.rs:38-55"""
    s = State.zero_state(2)
    before = float(np.sum(np.abs(s.vector()) ** 2))
    s.normalize()
    assert abs(float(np.sum(np.abs(s.vector()) ** 2)) - before) < TOL

"""GPU: the executed known answers of the reference's dense circuit tests
(tests/test_circuits_dense.rs) that the fixture does not hold: a
gates::matrix X through add_operation, composition, reversal and
execute_and_measure (seeded draws here; the reference draws 100 times)."""
import pytest

from logosq_b200 import Circuit, State
from logosq_b200.gates import x_gate

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_execute_circuit():
    """tests/test_circuits_dense.rs:63-78"""
    c = Circuit(1)
    c.add_operation(x_gate(), [0], "X on 0")
    st = State.zero_state(1)
    c.execute(st)
    assert st.probability(0) < TOL and abs(st.probability(1) - 1.0) < TOL


def test_composition_executes_both():
    """tests/test_circuits_dense.rs:80-104"""
    a, b = Circuit(2), Circuit(2)
    a.x(0)
    b.h(1)
    a.compose(b)
    st = State.zero_state(2)
    a.execute(st)
    assert st.probability(0) < TOL and st.probability(1) < TOL
    assert abs(st.probability(2) - 0.5) < TOL and abs(st.probability(3) - 0.5) < TOL


def test_reversal_probabilities():
    """tests/test_circuits_dense.rs:106-133"""
    c = Circuit(1)
    c.x(0).h(0)
    for circ in (c, c.reversed()):
        st = State.zero_state(1)
        circ.execute(st)
        assert abs(st.probability(0) - 0.5) < TOL and abs(st.probability(1) - 0.5) < TOL


def test_execute_and_measure():
    """tests/test_circuits_dense.rs:800-830"""
    c = Circuit(1)
    c.x(0)
    r = c.execute_and_measure()
    assert len(r) == 1 and r[0] == 1
    h = Circuit(1)
    h.h(0)
    ones = sum(h.execute_and_measure(seed=s)[0] for s in range(100))
    assert 30 < ones < 70 and 30 < 100 - ones < 70

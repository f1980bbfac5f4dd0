"""GPU: the remaining known answers of the reference's QFT and normalisation
tests through the engine: qft::apply on |00> (tests/test_qft.rs:43-58), the
controlled phase on a uniform superposition (tests/test_qft.rs:167-187) and
State::new against a manual normalisation (tests/test_normalize.rs:125-150)."""
import math

import numpy as np
import pytest

from logosq_b200 import Circuit, State, qft

pytestmark = pytest.mark.gpu


def test_qft_apply_on_zero_state():
    """tests/test_qft.rs:43-58 (epsilon 1e-5, as the reference)"""
    st = State.zero_state(2)
    qft.apply(st)
    v = st.vector()
    assert np.abs(np.abs(v) - 1.0 / math.sqrt(len(v))).max() < 1e-5


@pytest.mark.parametrize("angle", [math.pi / 4, math.pi / 2, math.pi])
def test_controlled_phase_keeps_uniform_magnitudes(angle):
    """tests/test_qft.rs:167-187"""
    c = Circuit(2)
    qft.controlled_phase(c, 0, 1, angle)
    c.h(0)
    c.h(1)
    st = State.zero_state(2)
    c.execute(st)
    assert np.abs(np.abs(st.vector()) - 0.5).max() < 1e-5


def test_normalize_against_manual():
    """tests/test_normalize.rs:125-150"""
    vec = np.array([complex(((i * 17) % 100) / 50.0 - 1.0, ((i * 23) % 100) / 50.0 - 1.0)
                    for i in range(16)])
    st = State.new(vec, 4)
    want = vec / math.sqrt(float(np.sum(np.abs(vec) ** 2)))
    assert np.abs(st.vector() - want).max() < 1e-10


def test_normalize_plus_state():
    """tests/test_normalize.rs:106-122 (normalising a normalised state keeps it)"""
    st = State.plus_state(4)
    st.normalize()
    assert np.abs(st.vector() - 0.25).max() < 1e-12

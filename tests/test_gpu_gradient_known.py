"""GPU: every test of the reference's gradient file
(tests/test_optimization_gradient.rs) through the engine's ParameterShift and
FiniteDifference (src/optimization/gradient.rs:22-126), with the reference's
parameters and thresholds."""
import math

import numpy as np
import pytest

from logosq_b200 import (EntanglingGate, EntanglingPattern, FiniteDifference,
                         HardwareEfficientAnsatz, ParameterShift, Pauli, PauliObservable,
                         PauliTerm, RealAmplitudesAnsatz)

pytestmark = pytest.mark.gpu
PI = math.pi


def hea(n, depth):
    return HardwareEfficientAnsatz(n, depth, EntanglingGate.CNOT, EntanglingPattern.Linear)


def obs_of(n, terms):
    o = PauliObservable(n)
    for c, p in terms:
        o.add_term(PauliTerm(c, p))
    return o


def test_parameter_shift_simple():
    """tests/test_optimization_gradient.rs:14-35"""
    g = ParameterShift.new().compute_gradient(hea(1, 1), PauliObservable.single_z(1, 0),
                                              [PI / 4, PI / 6])
    assert len(g) == 2 and np.any(np.abs(g) > 1e-10)


def test_parameter_shift_at_extremum():
    """tests/test_optimization_gradient.rs:37-60"""
    g = ParameterShift.new().compute_gradient(hea(1, 1), PauliObservable.single_z(1, 0),
                                              [0.0, 0.0])
    assert len(g) == 2 and np.all(np.abs(g) < 1e-8)


def test_parameter_shift_known_value():
    """tests/test_optimization_gradient.rs:62-89"""
    g = ParameterShift.new().compute_gradient(hea(1, 0), PauliObservable.single_z(1, 0),
                                              [PI / 4])
    assert abs(g[0] + math.sin(PI / 4)) < 1e-6


def test_parameter_shift_vs_finite_difference():
    """tests/test_optimization_gradient.rs:91-114"""
    a, o = RealAmplitudesAnsatz(2, 1), PauliObservable.single_z(2, 0)
    p = [0.5, 1.0, 1.5, 0.3, 0.8, 0.2]
    ps = ParameterShift.new().compute_gradient(a, o, p)
    fd = FiniteDifference(1e-5).compute_gradient(a, o, p)
    assert np.abs(ps - fd).max() < 1e-4


def test_gradient_at_minimum():
    """tests/test_optimization_gradient.rs:116-137"""
    g = ParameterShift.new().compute_gradient(hea(1, 1), PauliObservable.single_z(1, 0),
                                              [PI, 0.0])
    assert np.all(np.abs(g) < 0.1)


def test_finite_difference_custom_epsilon():
    """tests/test_optimization_gradient.rs:139-165"""
    a, o, p = RealAmplitudesAnsatz(1, 1), PauliObservable.single_z(1, 0), [0.5, 1.0]
    gl = FiniteDifference(1e-3).compute_gradient(a, o, p)
    gs = FiniteDifference(1e-7).compute_gradient(a, o, p)
    assert len(gl) == len(gs) == 2 and np.abs(gl - gs).max() < 1e-3


def test_parameter_shift_custom_shift():
    """tests/test_optimization_gradient.rs:167-190"""
    a, o, p = hea(1, 1), PauliObservable.single_z(1, 0), [0.5, 1.0]
    gd = ParameterShift.new().compute_gradient(a, o, p)
    gc = ParameterShift.with_shift(PI / 4).compute_gradient(a, o, p)
    assert len(gd) == len(gc) and np.all(np.isfinite(gd)) and np.all(np.isfinite(gc))


def test_gradient_two_qubit_system():
    """tests/test_optimization_gradient.rs:192-211"""
    g = ParameterShift.new().compute_gradient(hea(2, 1), PauliObservable.zz_interaction(2, 0, 1, 1.0),
                                              [0.2, 0.4, 0.6, 0.8])
    assert len(g) == 4 and np.sum(np.abs(g)) > 1e-10


def test_gradient_linearity():
    """tests/test_optimization_gradient.rs:213-240"""
    a, p = RealAmplitudesAnsatz(2, 1), [0.5, 1.0, 1.5, 0.3, 0.8, 0.2]
    g1 = ParameterShift.new().compute_gradient(a, PauliObservable.single_z(2, 0), p)
    g2 = ParameterShift.new().compute_gradient(a, obs_of(2, [(2.0, [Pauli.Z, Pauli.I])]), p)
    assert np.abs(g2 - 2.0 * g1).max() < 1e-10


def test_gradient_vanishes_for_identity():
    """tests/test_optimization_gradient.rs:242-264"""
    g = ParameterShift.new().compute_gradient(hea(2, 1), obs_of(2, [(1.0, [Pauli.I, Pauli.I])]),
                                              [0.5, 1.0, 1.5, 2.0])
    assert np.all(np.abs(g) < 1e-10)


def test_gradient_symmetry():
    """tests/test_optimization_gradient.rs:266-299"""
    o = obs_of(2, [(1.0, [Pauli.Z, Pauli.I]), (1.0, [Pauli.I, Pauli.Z])])
    g = ParameterShift.new().compute_gradient(hea(2, 1), o, [0.5] * 4)
    assert len(g) == 4 and abs(g[0] - g[1]) < 1e-6


def test_gradient_multiple_observables():
    """tests/test_optimization_gradient.rs:301-318"""
    o = obs_of(2, [(0.5, [Pauli.Z, Pauli.I]), (1.0, [Pauli.Z, Pauli.Z])])
    p = [0.3, 0.7, 1.1, 0.5, 0.9, 1.3]
    g = ParameterShift.new().compute_gradient(RealAmplitudesAnsatz(2, 1), o, p)
    assert len(g) == len(p) and np.any(np.abs(g) > 1e-10)

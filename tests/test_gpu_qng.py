"""GPU: QuantumNaturalGradient (src/optimization/qng.rs) on the engine against
the same formula evaluated on oracle states (1e-12), and the reference's
placeholder solve (the natural gradient equals the plain gradient)."""
import numpy as np
import pytest

import oracle
from logosq_b200 import (HardwareEfficientAnsatz, ParameterShift, PauliObservable,
                         QuantumNaturalGradient, VariationalQuantumCircuit, workloads)

pytestmark = pytest.mark.gpu


def oracle_metric(ansatz, theta, reg):
    n = ansatz.num_qubits()
    tpl = ansatz.template().packed()
    P = len(theta)
    s = np.pi / 2

    def state(v):
        return oracle.apply_circuit(oracle.zero_state(n), tpl, v)

    g = np.zeros((P, P))
    for i in range(P):
        for j in range(i, P):
            vs = []
            for si, sj in ((1, 1), (1, -1), (-1, 1), (-1, -1)):
                v = theta.copy()
                v[i] += si * s
                v[j] += sj * s
                vs.append(state(v))
            pp, pm, mp, mm = vs
            val = (abs(np.vdot(pp, pp)) - abs(np.vdot(pp, pm)) - abs(np.vdot(mp, pp)) +
                   abs(np.vdot(mm, mm))) / 8
            g[i, j] = g[j, i] = val
    return g + reg * np.eye(P)


@pytest.mark.parametrize("make", [lambda: HardwareEfficientAnsatz(4, 1),
                                  lambda: VariationalQuantumCircuit(3, 2)])
def test_metric_tensor_matches_oracle(make):
    a = make()
    theta = np.random.default_rng(3).uniform(-np.pi, np.pi, a.num_parameters())
    got = QuantumNaturalGradient().compute_metric_tensor(a, theta)
    want = oracle_metric(a, theta, 1e-8)
    assert np.abs(got - want).max() < 1e-12
    assert np.allclose(got, got.T)


def test_natural_gradient_is_the_plain_gradient():
    a = VariationalQuantumCircuit(3, 2)
    theta = np.random.default_rng(5).uniform(-np.pi, np.pi, a.num_parameters())
    obs = PauliObservable(3)
    terms = workloads.heisenberg_terms(3, [0.4, -0.7], [0.2, 0.5], [1.0, -0.3], 0.1)
    obs._packed = terms
    obs.terms = [None] * len(terms)
    qng = QuantumNaturalGradient.with_regularization(1e-6)
    got = qng.compute_natural_gradient(a, obs, ParameterShift(), theta)
    want = ParameterShift().compute_gradient(a, obs, theta)
    assert np.array_equal(np.asarray(got), np.asarray(want))

"""CPU: the reference's optimizer tests (tests/test_optimization.rs:16-154) on
classical objectives through the mirror's GradientDescent and Adam
(src/optimization/optimizer.rs:57-223), with the reference's builder calls and
tolerances."""
from logosq_b200 import LBFGSB, Adam, GradientDescent


def test_gradient_descent_simple_quadratic():
    """tests/test_optimization.rs:16-30"""
    r = GradientDescent(0.1, 100).with_tolerance(1e-6).minimize(
        lambda x: x[0] * x[0], lambda x: [2.0 * x[0]], [5.0])
    assert r.converged
    assert abs(r.optimal_parameters[0]) < 0.1 and r.optimal_value < 0.01


def test_gradient_descent_two_variables():
    """tests/test_optimization.rs:32-46"""
    r = GradientDescent(0.1, 100).with_tolerance(1e-6).minimize(
        lambda p: p[0] * p[0] + p[1] * p[1], lambda p: [2.0 * p[0], 2.0 * p[1]], [3.0, 4.0])
    assert r.converged
    assert abs(r.optimal_parameters[0]) < 0.1 and abs(r.optimal_parameters[1]) < 0.1


def _shifted(p):
    return (p[0] - 1.0) ** 2 + (p[1] + 2.0) ** 2


def _shifted_grad(p):
    return [2.0 * (p[0] - 1.0), 2.0 * (p[1] + 2.0)]


def test_adam_optimizer():
    """tests/test_optimization.rs:48-62"""
    r = Adam(0.1, 200).with_tolerance(1e-6).minimize(_shifted, _shifted_grad, [5.0, 5.0])
    assert r.converged
    assert abs(r.optimal_parameters[0] - 1.0) < 0.1
    assert abs(r.optimal_parameters[1] + 2.0) < 0.1


def test_adam_converges_on_1d_quadratic():
    """tests/test_optimization.rs:64-76"""
    r = Adam(0.1, 200).with_tolerance(1e-6).minimize(
        lambda p: (p[0] - 3.0) ** 2, lambda p: [2.0 * (p[0] - 3.0)], [10.0])
    assert r.converged
    assert abs(r.optimal_parameters[0] - 3.0) < 1e-3 and r.optimal_value < 1e-6


def test_adam_converges_on_shifted_2d_quadratic():
    """tests/test_optimization.rs:78-94"""
    r = Adam(0.1, 200).with_tolerance(1e-6).minimize(_shifted, _shifted_grad, [5.0, 5.0])
    assert r.converged
    assert abs(r.optimal_parameters[0] - 1.0) < 1e-2
    assert abs(r.optimal_parameters[1] + 2.0) < 1e-2
    assert r.optimal_value < 1e-4


def test_adam_gradient_norm_convergence():
    """tests/test_optimization.rs:96-109"""
    r = Adam(0.2, 100).with_tolerance(1e-6).minimize(
        lambda p: sum(x * x for x in p), lambda p: [2.0 * x for x in p], [1e-3, -1e-3])
    assert r.converged


def test_adam_small_step_convergence():
    """tests/test_optimization.rs:111-124"""
    r = Adam(0.1, 100).with_tolerance(1e-6).minimize(
        lambda p: 1.0 + 1e-8 * p[0] * p[0], lambda p: [2.0e-8 * p[0]], [1.0])
    assert r.converged


def test_convergence_history_decreases():
    """tests/test_optimization.rs:126-138"""
    r = GradientDescent(0.1, 50).minimize(lambda x: x[0] * x[0], lambda x: [2.0 * x[0]], [10.0])
    h = r.convergence_history
    assert all(h[i] <= h[i - 1] for i in range(1, len(h)))


def test_max_iterations():
    """tests/test_optimization.rs:140-154"""
    r = GradientDescent(0.001, 10).minimize(lambda x: x[0] * x[0], lambda x: [2.0 * x[0]],
                                            [100.0])
    assert r.num_iterations <= 10


def test_lbfgsb_interface():
    """LBFGSB::new (src/optimization/optimizer.rs:233-241): settings only."""
    o = LBFGSB(50)
    assert (o.max_iterations, o.tolerance, o.m) == (50, 1e-6, 10)

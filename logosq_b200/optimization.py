"""Variational layer: the drop-in for src/optimization/*.rs.

Observables are packed Pauli strings evaluated on the device in FP64
(lq_expectation_pauli).  Ansatz classes describe their circuit once as a
parameterised descriptor list (a "template"); ParameterShift and
FiniteDifference hand that template to the engine, which re-binds the angles
for every shifted circuit (lq_parameter_shift / lq_finite_difference).
"""
from __future__ import annotations

import ctypes as C
import enum
import math
from typing import Protocol, runtime_checkable

import numpy as np

from . import abi
from ._lib import LogosQError, call
from .circuits import Circuit
from .states import State


# ---------------------------------------------------------------------------
# Observables (src/optimization/observable.rs)
# ---------------------------------------------------------------------------
class Pauli(enum.Enum):
    I = 0
    X = 1
    Y = 2
    Z = 3

    def matrix(self):
        return {
            Pauli.I: np.eye(2, dtype=np.complex128),
            Pauli.X: np.array([[0, 1], [1, 0]], dtype=np.complex128),
            Pauli.Y: np.array([[0, -1j], [1j, 0]], dtype=np.complex128),
            Pauli.Z: np.array([[1, 0], [0, -1]], dtype=np.complex128),
        }[self]


class PauliTerm:
    """PauliTerm (src/optimization/observable.rs:79-147)."""

    def __init__(self, coefficient: float, paulis):
        self.coefficient = float(coefficient)
        self.paulis = list(paulis)

    def packed(self) -> tuple[int, int, int]:
        n = len(self.paulis)
        x = z = ny = 0
        for q, p in enumerate(self.paulis):
            b = 1 << (n - 1 - q)
            if p in (Pauli.X, Pauli.Y):
                x |= b
            if p in (Pauli.Z, Pauli.Y):
                z |= b
            if p is Pauli.Y:
                ny += 1
        return x, z, ny

    def expectation(self, state: State, y_convention: int = abi.Y_REFERENCE) -> float:
        if len(self.paulis) != state.num_qubits():
            raise LogosQError(abi.LQ_ERR_DIMENSION_MISMATCH,
                              "Pauli term must have operator for each qubit")
        return PauliObservable.from_terms(len(self.paulis), [self]).expectation(state, y_convention)


def pack_terms(terms, num_qubits: int) -> np.ndarray:
    arr = np.zeros(len(terms), dtype=abi.TERM_DTYPE)
    for i, t in enumerate(terms):
        if len(t.paulis) != num_qubits:
            raise LogosQError(abi.LQ_ERR_DIMENSION_MISMATCH,
                              "Term must match observable qubit count")
        x, z, ny = t.packed()
        arr[i]["coefficient"] = t.coefficient
        arr[i]["xmask"] = np.uint64(x)
        arr[i]["zmask"] = np.uint64(z)
        arr[i]["ny"] = ny
    return arr


class Observable:
    """Trait `Observable` (src/optimization/observable.rs:10-18)."""

    def expectation(self, state: State) -> float:  # pragma: no cover - abstract
        raise NotImplementedError


class PauliObservable(Observable):
    """PauliObservable (src/optimization/observable.rs:152-232)."""

    def __init__(self, num_qubits: int):
        self.num_qubits = int(num_qubits)
        self.terms: list[PauliTerm] = []
        self._packed = None
        self.y_convention = abi.Y_REFERENCE

    @classmethod
    def from_terms(cls, num_qubits, terms):
        o = cls(num_qubits)
        for t in terms:
            o.add_term(t)
        return o

    def add_term(self, term: PauliTerm) -> None:
        if len(term.paulis) != self.num_qubits:
            raise LogosQError(abi.LQ_ERR_DIMENSION_MISMATCH,
                              "Term must match observable qubit count")
        self.terms.append(term)
        self._packed = None

    def packed(self) -> np.ndarray:
        if self._packed is None:
            self._packed = pack_terms(self.terms, self.num_qubits)
        return self._packed

    @staticmethod
    def _check_qubit(q, num_qubits):
        # The reference asserts "Qubit index out of bounds" (observable.rs:177, 193-194, 210).
        if not 0 <= q < num_qubits:
            raise LogosQError(abi.LQ_ERR_QUBIT_INDEX, "Qubit index out of bounds")

    @classmethod
    def single_z(cls, num_qubits, target_qubit):
        cls._check_qubit(target_qubit, num_qubits)
        p = [Pauli.I] * num_qubits
        p[target_qubit] = Pauli.Z
        return cls.from_terms(num_qubits, [PauliTerm(1.0, p)])

    @classmethod
    def zz_interaction(cls, num_qubits, qubit1, qubit2, coefficient):
        cls._check_qubit(qubit1, num_qubits)
        cls._check_qubit(qubit2, num_qubits)
        p = [Pauli.I] * num_qubits
        p[qubit1] = Pauli.Z
        p[qubit2] = Pauli.Z
        return cls.from_terms(num_qubits, [PauliTerm(coefficient, p)])

    @classmethod
    def ising_hamiltonian(cls, num_qubits, j_couplings, h_fields):
        o = cls(num_qubits)
        for i, j in enumerate(j_couplings):
            cls._check_qubit(i + 1, num_qubits)
            p = [Pauli.I] * num_qubits
            p[i] = Pauli.Z
            p[i + 1] = Pauli.Z
            o.add_term(PauliTerm(j, p))
        for i, hf in enumerate(h_fields):
            cls._check_qubit(i, num_qubits)
            p = [Pauli.I] * num_qubits
            p[i] = Pauli.Z
            o.add_term(PauliTerm(hf, p))
        return o

    def expectation(self, state: State, y_convention: int | None = None) -> float:
        yc = self.y_convention if y_convention is None else y_convention
        t = self.packed()
        out = C.c_double()
        call("lq_expectation_pauli", state.handle, abi.term_ptr(t), len(t), yc, C.byref(out), None)
        return out.value

    def term_expectations(self, state: State) -> np.ndarray:
        t = self.packed()
        out = C.c_double()
        per = np.zeros(len(t), dtype=np.float64)
        call("lq_expectation_pauli", state.handle, abi.term_ptr(t), len(t), self.y_convention,
             C.byref(out), abi.f64_ptr(per))
        return per


# ---------------------------------------------------------------------------
# Ansatz (src/optimization/ansatz.rs, src/qml/vqc.rs)
# ---------------------------------------------------------------------------
class Ansatz:
    """Trait `Ansatz` (src/optimization/ansatz.rs:10-43).

    Subclasses implement `template()`: the circuit with every angle bound to a
    parameter index, so that build_circuit(params) = template with params.
    """

    def num_parameters(self) -> int:  # pragma: no cover - abstract
        raise NotImplementedError

    def num_qubits(self) -> int:  # pragma: no cover - abstract
        raise NotImplementedError

    def template(self) -> Circuit:  # pragma: no cover - abstract
        raise NotImplementedError

    def build_circuit(self, parameters) -> Circuit:
        """A concrete circuit (angles substituted on the host)."""
        p = np.asarray(parameters, dtype=np.float64)
        if len(p) != self.num_parameters():
            raise LogosQError(abi.LQ_ERR_PARAM_COUNT,
                              f"Parameter count mismatch: expected {self.num_parameters()}, "
                              f"got {len(p)}")
        tpl = self.template().packed().copy()
        for k in range(3):
            sel = tpl["param"][:, k] >= 0
            idx = tpl["param"][sel, k]
            tpl["angle"][sel, k] = p[idx] * tpl["scale"][sel, k] + tpl["angle"][sel, k]
            tpl["param"][sel, k] = -1
        c = Circuit(self.num_qubits())
        for rec in tpl:
            c._push(rec.reshape(1).copy(), [q for q in rec["q"] if q >= 0], "op")
        return c

    def apply(self, state: State, parameters) -> None:
        """Ansatz::apply (src/optimization/ansatz.rs:21-37)."""
        if state.num_qubits() != self.num_qubits():
            raise LogosQError(abi.LQ_ERR_QUBIT_MISMATCH, "State qubit count must match ansatz")
        p = np.ascontiguousarray(parameters, dtype=np.float64)
        if len(p) != self.num_parameters():
            raise LogosQError(abi.LQ_ERR_PARAM_COUNT,
                              f"Parameter count mismatch: expected {self.num_parameters()}, "
                              f"got {len(p)}")
        self.template().execute(state, theta=p)

    def parameter_bounds(self):
        return None


class AnsatzType(enum.Enum):
    """AnsatzType (src/optimization/ansatz.rs:45-56)."""
    HardwareEfficient = 0
    RealAmplitudes = 1
    EfficientSU2 = 2
    Custom = 3


class EntanglingGate(enum.Enum):
    CNOT = "cnot"
    CZ = "cz"
    RZZ = "rzz"


class EntanglingPattern(enum.Enum):
    Linear = 0
    Circular = 1
    Full = 2


class HardwareEfficientAnsatz(Ansatz):
    """HardwareEfficientAnsatz (src/optimization/ansatz.rs:63-186)."""

    def __init__(self, num_qubits, depth, entangling_gate=EntanglingGate.CNOT,
                 entangling_pattern=EntanglingPattern.Linear, rzz_angle=0.0):
        self.n, self.depth = int(num_qubits), int(depth)
        self.entangling_gate, self.entangling_pattern = entangling_gate, entangling_pattern
        self.rzz_angle = rzz_angle
        self._tpl = None

    def num_parameters(self):
        return self.n * (self.depth + 1)

    def num_qubits(self):
        return self.n

    def parameter_bounds(self):
        return [(0.0, 2.0 * math.pi)] * self.num_parameters()

    def _ent(self, c, i, j):
        if self.entangling_gate is EntanglingGate.CNOT:
            c.cnot(i, j)
        elif self.entangling_gate is EntanglingGate.CZ:
            c.cz(i, j)
        else:
            c.rzz(i, j, self.rzz_angle)

    def _ent_layer(self, c):
        n = self.n
        if self.entangling_pattern is EntanglingPattern.Linear:
            for i in range(n - 1):
                self._ent(c, i, i + 1)
        elif self.entangling_pattern is EntanglingPattern.Circular:
            for i in range(n - 1):
                self._ent(c, i, i + 1)
            if n > 2:
                self._ent(c, n - 1, 0)
        else:
            for i in range(n):
                for j in range(i + 1, n):
                    self._ent(c, i, j)

    def template(self):
        if self._tpl is None:
            c, p = Circuit(self.n), 0
            for layer in range(self.depth):
                for q in range(self.n):
                    c.ry_param(q, p)
                    p += 1
                if layer < self.depth - 1 or self.depth == 1:
                    self._ent_layer(c)
            for q in range(self.n):
                c.ry_param(q, p)
                p += 1
            self._tpl = c
        return self._tpl


class RealAmplitudesAnsatz(Ansatz):
    """RealAmplitudesAnsatz (src/optimization/ansatz.rs:190-248)."""

    def __init__(self, num_qubits, depth):
        self.n, self.depth = int(num_qubits), int(depth)
        self._tpl = None

    def num_parameters(self):
        if self.n > 1 and self.depth == 1:
            return self.n * (self.depth + 2)
        return self.n * (self.depth + 1)

    def num_qubits(self):
        return self.n

    def template(self):
        if self._tpl is None:
            c, p = Circuit(self.n), 0
            if self.n > 1 and self.depth == 1:
                for q in range(self.n):
                    c.ry_param(q, p)
                    p += 1
            for _ in range(self.depth):
                for q in range(self.n):
                    c.ry_param(q, p)
                    p += 1
                for i in range(self.n - 1):
                    c.cnot(i, i + 1)
            for q in range(self.n):
                c.ry_param(q, p)
                p += 1
            self._tpl = c
        return self._tpl


class EfficientSU2Ansatz(Ansatz):
    """EfficientSU2Ansatz (src/optimization/ansatz.rs:252-294)."""

    def __init__(self, num_qubits, depth):
        self.n, self.depth = int(num_qubits), int(depth)
        self._tpl = None

    def num_parameters(self):
        return 3 * self.n * self.depth

    def num_qubits(self):
        return self.n

    def template(self):
        if self._tpl is None:
            c, p = Circuit(self.n), 0
            for _ in range(self.depth):
                for q in range(self.n):
                    c.rz_param(q, p)
                    c.ry_param(q, p + 1)
                    c.rz_param(q, p + 2)
                    p += 3
                for i in range(self.n - 1):
                    c.cnot(i, i + 1)
            self._tpl = c
        return self._tpl


class ParameterizedCircuit(Ansatz):
    """ParameterizedCircuit (src/optimization/ansatz.rs:298-335): a user builder
    closure params -> Circuit.  Without a template, each evaluation builds and
    executes a concrete circuit."""

    def __init__(self, num_qubits, num_parameters, builder):
        self.n, self.p, self.builder = int(num_qubits), int(num_parameters), builder

    def num_parameters(self):
        return self.p

    def num_qubits(self):
        return self.n

    def template(self):
        raise LogosQError(abi.LQ_ERR_UNSUPPORTED, "ParameterizedCircuit has no template")

    def build_circuit(self, parameters):
        return self.builder(np.asarray(parameters, dtype=np.float64))

    def apply(self, state, parameters):
        self.build_circuit(parameters).execute(state)


def _energy_closure(ansatz, observable):
    """The VQE objective (src/optimization/vqe.rs:63-67)."""
    work = State(ansatz.num_qubits())

    def f(params):
        p = np.ascontiguousarray(params, dtype=np.float64)
        if isinstance(observable, PauliObservable) and not isinstance(ansatz, ParameterizedCircuit):
            tpl = ansatz.template().packed()
            t = observable.packed()
            out = C.c_double()
            call("lq_ansatz_energy", work.handle, abi.gate_ptr(tpl), len(tpl), abi.f64_ptr(p),
                 len(p), abi.term_ptr(t), len(t), observable.y_convention, C.byref(out))
            return out.value
        call("lq_state_set_basis", work.handle, C.c_uint64(0))
        ansatz.apply(work, p)
        return observable.expectation(work)

    return f, work


# ---------------------------------------------------------------------------
# Gradients (src/optimization/gradient.rs)
# ---------------------------------------------------------------------------
class GradientMethod:
    def compute_gradient(self, ansatz, observable, parameters):  # pragma: no cover
        raise NotImplementedError


class ParameterShift(GradientMethod):
    """ParameterShift (src/optimization/gradient.rs:22-78)."""

    def __init__(self, shift: float = math.pi / 2.0):
        self.shift = float(shift)

    @classmethod
    def new(cls):
        return cls()

    @classmethod
    def with_shift(cls, shift):
        return cls(shift)

    def compute_gradient(self, ansatz, observable, parameters):
        p = np.ascontiguousarray(parameters, dtype=np.float64)
        if isinstance(observable, PauliObservable) and not isinstance(ansatz, ParameterizedCircuit):
            work = State(ansatz.num_qubits())
            tpl = ansatz.template().packed()
            t = observable.packed()
            g = np.zeros(len(p), dtype=np.float64)
            call("lq_parameter_shift", work.handle, abi.gate_ptr(tpl), len(tpl), abi.f64_ptr(p),
                 len(p), abi.term_ptr(t), len(t), observable.y_convention, self.shift,
                 abi.f64_ptr(g))
            work.close()
            return g
        f, work = _energy_closure(ansatz, observable)
        g = np.zeros(len(p))
        for i in range(len(p)):
            pp = p.copy()
            pp[i] += self.shift
            ep = f(pp)
            pp[i] = p[i] - self.shift
            em = f(pp)
            g[i] = (ep - em) / 2.0
        work.close()
        return g


class FiniteDifference(GradientMethod):
    """FiniteDifference (src/optimization/gradient.rs:81-126)."""

    def __init__(self, epsilon: float = 1e-7):
        self.epsilon = float(epsilon)

    def compute_gradient(self, ansatz, observable, parameters):
        p = np.ascontiguousarray(parameters, dtype=np.float64)
        if isinstance(observable, PauliObservable) and not isinstance(ansatz, ParameterizedCircuit):
            work = State(ansatz.num_qubits())
            tpl = ansatz.template().packed()
            t = observable.packed()
            g = np.zeros(len(p), dtype=np.float64)
            call("lq_finite_difference", work.handle, abi.gate_ptr(tpl), len(tpl),
                 abi.f64_ptr(p), len(p), abi.term_ptr(t), len(t), observable.y_convention,
                 self.epsilon, abi.f64_ptr(g))
            work.close()
            return g
        f, work = _energy_closure(ansatz, observable)
        fx = f(p)
        g = np.zeros(len(p))
        for i in range(len(p)):
            pp = p.copy()
            pp[i] += self.epsilon
            g[i] = (f(pp) - fx) / self.epsilon
        work.close()
        return g


# ---------------------------------------------------------------------------
# Optimizers and VQE (src/optimization/optimizer.rs, vqe.rs)
# ---------------------------------------------------------------------------
class OptimizerResult:
    def __init__(self, optimal_parameters, optimal_value, num_iterations, convergence_history,
                 converged):
        self.optimal_parameters = optimal_parameters
        self.optimal_value = optimal_value
        self.num_iterations = num_iterations
        self.convergence_history = convergence_history
        self.converged = converged


@runtime_checkable
class Optimizer(Protocol):
    """Trait Optimizer (src/optimization/optimizer.rs:17-33); GradientDescent and
    Adam satisfy it."""

    def minimize(self, f, grad_f, initial_params) -> "OptimizerResult": ...


class GradientDescent:
    """GradientDescent::minimize (src/optimization/optimizer.rs:57-107)."""

    def __init__(self, learning_rate, max_iterations, tolerance=1e-6, verbose=False):
        self.learning_rate, self.max_iterations = learning_rate, max_iterations
        self.tolerance, self.verbose = tolerance, verbose

    def with_tolerance(self, tolerance) -> "GradientDescent":
        """GradientDescent::with_tolerance (src/optimization/optimizer.rs:50-53)."""
        self.tolerance = tolerance
        return self

    def minimize(self, f, grad_f, initial_params):
        params = np.array(initial_params, dtype=np.float64)
        hist, converged = [], False
        for it in range(self.max_iterations):
            value = f(params)
            hist.append(value)
            g = np.asarray(grad_f(params))
            gn = math.sqrt(float(np.sum(g * g)))
            if gn < self.tolerance:
                converged = True
                break
            for i in range(len(params)):
                params[i] -= self.learning_rate * g[i]
            if self.verbose and it % 10 == 0:
                print(f"Iteration {it}: value = {value:.6f}, |grad| = {gn:.6f}")
        opt = f(params)
        fg = np.asarray(grad_f(params))
        if math.sqrt(float(np.sum(fg * fg))) < self.tolerance:
            converged = True
        return OptimizerResult(params, opt, len(hist), hist, converged)


class Adam:
    """Adam::minimize (src/optimization/optimizer.rs:139-223)."""

    def __init__(self, learning_rate, max_iterations, tolerance=1e-6, verbose=False):
        self.learning_rate, self.max_iterations = learning_rate, max_iterations
        self.beta1, self.beta2, self.epsilon = 0.9, 0.999, 1e-8
        self.tolerance, self.verbose = tolerance, verbose

    def with_tolerance(self, tolerance) -> "Adam":
        """Adam::with_tolerance (src/optimization/optimizer.rs:132-135)."""
        self.tolerance = tolerance
        return self

    def minimize(self, f, grad_f, initial_params):
        params = np.array(initial_params, dtype=np.float64)
        n = len(params)
        m, v = [0.0] * n, [0.0] * n
        hist, converged, prev = [], False, None
        for it in range(1, self.max_iterations + 1):
            value = f(params)
            hist.append(value)
            if prev is not None and abs(prev - value) < self.tolerance:
                converged = True
                break
            prev = value
            g = np.asarray(grad_f(params))
            gn = math.sqrt(float(np.sum(g * g)))
            if gn < self.tolerance:
                converged = True
                break
            for i in range(n):
                m[i] = self.beta1 * m[i] + (1.0 - self.beta1) * g[i]
                v[i] = self.beta2 * v[i] + (1.0 - self.beta2) * g[i] * g[i]
            mc = 1.0 / (1.0 - self.beta1 ** it)
            vc = 1.0 / (1.0 - self.beta2 ** it)
            step_sq = 0.0
            for i in range(n):
                step = self.learning_rate * (m[i] * mc) / (math.sqrt(v[i] * vc) + self.epsilon)
                params[i] -= step
                step_sq += step * step
            if math.sqrt(step_sq) < self.tolerance:
                converged = True
                break
            if self.verbose and it % 10 == 0:
                print(f"Iteration {it}: value = {value:.6f}, |grad| = {gn:.6f}")
        opt = f(params)
        fg = np.asarray(grad_f(params))
        if math.sqrt(float(np.sum(fg * fg))) < self.tolerance:
            converged = True
        return OptimizerResult(params, opt, len(hist), hist, converged)


class LBFGSB:
    """LBFGSB (src/optimization/optimizer.rs:227-241): the reference declares
    the optimizer's settings (iterations, tolerance 1e-6, memory 10) and no
    minimisation routine; the mirror keeps the same interface."""

    def __init__(self, max_iterations):
        self.max_iterations, self.tolerance, self.m = max_iterations, 1e-6, 10


class VQEResult:
    def __init__(self, ground_state_energy, optimal_parameters, num_iterations,
                 convergence_history, final_state):
        self.ground_state_energy = ground_state_energy
        self.optimal_parameters = optimal_parameters
        self.num_iterations = num_iterations
        self.convergence_history = convergence_history
        self.final_state = final_state


class VQE:
    """VQE (src/optimization/vqe.rs:22-111)."""

    def __init__(self, ansatz, hamiltonian, gradient_method, optimizer, verbose=False):
        self.ansatz, self.hamiltonian = ansatz, hamiltonian
        self.gradient_method, self.optimizer = gradient_method, optimizer
        self.verbose = verbose

    def run(self, initial_parameters) -> VQEResult:
        f, work = _energy_closure(self.ansatz, self.hamiltonian)

        def grad(params):
            return self.gradient_method.compute_gradient(self.ansatz, self.hamiltonian, params)

        res = self.optimizer.minimize(f, grad, initial_parameters)
        work.close()
        final = State.zero_state(self.ansatz.num_qubits())
        self.ansatz.apply(final, res.optimal_parameters)
        return VQEResult(res.optimal_value, res.optimal_parameters, res.num_iterations,
                         res.convergence_history, final)

    def run_random(self, seed: int = 0) -> VQEResult:
        rng = np.random.default_rng(seed)
        init = rng.uniform(0.0, 2.0 * math.pi, self.ansatz.num_parameters())
        return self.run(init)


# ---------------------------------------------------------------------------
# Quantum natural gradient (src/optimization/qng.rs)
# ---------------------------------------------------------------------------
class QuantumNaturalGradient:
    """QuantumNaturalGradient (src/optimization/qng.rs:12-141) on the device.

    compute_metric_tensor follows the reference's formula (qng.rs:29-87): for
    every pair i <= j the four states with parameters i, j shifted by
    (+s, +s), (+s, -s), (-s, +s), (-s, -s), s = pi/2, are prepared by the
    engine and
        g_ij = (|<pp|pp>| - |<pp|pm>| - |<mp|pp>| + |<mm|mm>|) / 8,
    symmetric, plus `regularization` on the diagonal.  States for a parameter
    vector that occurs more than once are prepared once.
    compute_natural_gradient returns the plain gradient, as the reference does:
    its linear solve is a placeholder that returns the right-hand side
    (qng.rs:117-134)."""

    def __init__(self, regularization: float = 1e-8):
        self.regularization = float(regularization)

    @classmethod
    def with_regularization(cls, regularization: float) -> "QuantumNaturalGradient":
        return cls(regularization)

    def compute_metric_tensor(self, ansatz, parameters) -> np.ndarray:
        p = np.asarray(parameters, dtype=np.float64)
        n = len(p)
        shift = math.pi / 2.0
        cache: dict = {}

        def state_for(vec):
            key = vec.tobytes()
            st = cache.get(key)
            if st is None:
                st = State.zero_state(ansatz.num_qubits())
                ansatz.apply(st, vec)
                cache[key] = st
            return st

        metric = np.zeros((n, n))
        try:
            for i in range(n):
                for j in range(i, n):
                    vecs = []
                    for si, sj in ((1, 1), (1, -1), (-1, 1), (-1, -1)):
                        v = p.copy()
                        v[i] += si * shift
                        v[j] += sj * shift
                        vecs.append(v)
                    pp, pm, mp, mm = (state_for(v) for v in vecs)
                    o_pp = abs(pp.inner_product(pp))
                    o_pm = abs(pp.inner_product(pm))
                    o_mp = abs(mp.inner_product(pp))
                    o_mm = abs(mm.inner_product(mm))
                    g = (o_pp - o_pm - o_mp + o_mm) / 8.0
                    metric[i, j] = g
                    metric[j, i] = g
                # states of row i are not needed again once j has passed them
                if len(cache) > 4 * (n + 1):
                    for st in cache.values():
                        st.close()
                    cache.clear()
        finally:
            for st in cache.values():
                st.close()
        metric[np.diag_indices(n)] += self.regularization
        return metric

    def compute_natural_gradient(self, ansatz, observable, gradient_method, parameters):
        gradient = np.asarray(gradient_method.compute_gradient(ansatz, observable, parameters))
        self.compute_metric_tensor(ansatz, parameters)
        return gradient

"""VariationalQuantumCircuit (src/qml/vqc.rs) as an Ansatz for the engine."""
from __future__ import annotations

import enum
import math

from . import abi
from ._lib import LogosQError
from .circuits import Circuit
from .optimization import Ansatz


class VQCType(enum.Enum):
    Simple = 0
    StronglyEntangling = 1
    BasicEntangling = 2
    Custom = 3


class VariationalQuantumCircuit(Ansatz):
    """VariationalQuantumCircuit (src/qml/vqc.rs:75-243).

    As an Ansatz the reference builds the circuit with empty inputs
    (src/qml/vqc.rs:230-243), so the input-encoding layer is absent there too.
    BasicEntangling (the default) is, per layer, RY(q) RZ(q) on every qubit and
    a CNOT(i, i+1) ladder: P = 2 n L parameters.
    """

    def __init__(self, num_qubits, num_layers, vqc_type=VQCType.BasicEntangling,
                 include_input_encoding=True):
        self.n, self.layers = int(num_qubits), int(num_layers)
        self.vqc_type = vqc_type
        self.include_input_encoding = include_input_encoding
        self._tpl = None

    @classmethod
    def new(cls, num_qubits, num_layers) -> "VariationalQuantumCircuit":
        """VariationalQuantumCircuit::new (src/qml/vqc.rs:84-91): BasicEntangling
        with the input-encoding layer."""
        return cls(num_qubits, num_layers)

    @property
    def num_layers(self):
        return self.layers

    def num_input_params(self):
        return self.n if self.include_input_encoding else 0

    def num_variational_params(self):
        if self.vqc_type is VQCType.Simple:
            return self.n * self.layers
        if self.vqc_type is VQCType.StronglyEntangling:
            return 3 * self.n * self.layers
        return 2 * self.n * self.layers

    def num_parameters(self):
        return self.num_variational_params()

    def num_qubits(self):
        return self.n

    def template(self, inputs=()):
        if inputs:
            return self._build(inputs)
        if self._tpl is None:
            self._tpl = self._build(())
        return self._tpl

    def _build(self, inputs):
        """build_circuit (src/qml/vqc.rs:117-171) with angles bound to params."""
        n = self.n
        c = Circuit(n)
        if self.include_input_encoding:
            for i, x in enumerate(list(inputs)[:n]):
                c.ry(i, math.pi * x)
        p = 0
        for layer in range(self.layers):
            if self.vqc_type is VQCType.Simple:
                for q in range(n):
                    c.ry_param(q, p)
                    p += 1
            elif self.vqc_type is VQCType.StronglyEntangling:
                for q in range(n):
                    c.rz_param(q, p)
                    c.ry_param(q, p + 1)
                    c.rz_param(q, p + 2)
                    p += 3
                offset = layer % n
                for i in range(max(n - 1, 0)):
                    ctl, tgt = (i + offset) % n, (i + 1 + offset) % n
                    if ctl != tgt:
                        c.cnot(ctl, tgt)
            else:
                for q in range(n):
                    c.ry_param(q, p)
                    c.rz_param(q, p + 1)
                    p += 2
                for i in range(max(n - 1, 0)):
                    c.cnot(i, i + 1)
        return c

    def forward(self, inputs, params):
        """forward (src/qml/vqc.rs:181-205): <Z> per qubit, where the reference
        reads bit `qubit` of the basis index (src/qml/vqc.rs:199-201)."""
        from .states import State
        from .optimization import PauliObservable, PauliTerm, Pauli
        st = State.zero_state(self.n)
        self._build(inputs).execute(st, theta=params)
        out = []
        for qubit in range(self.n):
            ps = [Pauli.I] * self.n
            ps[self.n - 1 - qubit] = Pauli.Z  # bit `qubit` is qubit n-1-qubit
            out.append(PauliObservable.from_terms(self.n, [PauliTerm(1.0, ps)]).expectation(st))
        return out

    def forward_activated(self, inputs, params):
        return [math.tanh(v) for v in self.forward(inputs, params)]


class VQCBuilder:
    """VQCBuilder (src/qml/vqc.rs:26-66): one layer, BasicEntangling and the
    input-encoding layer unless changed."""

    def __init__(self, num_qubits):
        self._n, self._layers = num_qubits, 1
        self._type, self._encoding = VQCType.BasicEntangling, True

    @classmethod
    def new(cls, num_qubits) -> "VQCBuilder":
        return cls(num_qubits)

    def with_layers(self, num_layers) -> "VQCBuilder":
        self._layers = num_layers
        return self

    def with_type(self, vqc_type) -> "VQCBuilder":
        self._type = vqc_type
        return self

    def with_input_encoding(self, include) -> "VQCBuilder":
        self._encoding = bool(include)
        return self

    def build(self) -> VariationalQuantumCircuit:
        return VariationalQuantumCircuit(self._n, self._layers, self._type, self._encoding)


class DressedVQC:
    """DressedVQC (src/qml/vqc.rs:251-284): a VQC with a per-output weight
    (1.0) and bias (0.0) applied to its outputs."""

    def __init__(self, vqc: VariationalQuantumCircuit, output_size: int):
        self.vqc = vqc
        self.output_weights = [1.0] * output_size
        self.output_biases = [0.0] * output_size

    def forward(self, inputs, params):
        return [v * w + b for v, w, b in zip(self.vqc.forward(inputs, params),
                                             self.output_weights, self.output_biases)]

    def num_params(self):
        return (self.vqc.num_variational_params() + len(self.output_weights)
                + len(self.output_biases))


def check_params(vqc: VariationalQuantumCircuit, params):
    if len(params) != vqc.num_parameters():
        raise LogosQError(abi.LQ_ERR_PARAM_COUNT,
                          f"Parameter count mismatch: expected {vqc.num_parameters()}, "
                          f"got {len(params)}")

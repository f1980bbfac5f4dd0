"""Device-resident quantum state: the drop-in for `State` (src/states/mod.rs:38-365).

The amplitudes live in HBM (complex128 by default); every method is a kernel
launch or a transfer through the C ABI.  Qubit q is bit (n-1-q) of the basis
index, as in the reference.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from typing import Protocol, runtime_checkable

from . import abi
from ._lib import LogosQError, call, lib


@runtime_checkable
class QuantumStateBackend(Protocol):
    """Trait QuantumStateBackend (src/states/backend.rs:14-60); State satisfies it."""

    def num_qubits(self) -> int: ...
    def apply_single_qubit_matrix(self, qubit, matrix) -> None: ...
    def apply_two_qubit_matrix(self, control, target, matrix) -> None: ...
    def apply_three_qubit_matrix(self, q1, q2, q3, matrix) -> None: ...
    def apply_full_matrix(self, matrix) -> None: ...


class State:
    """Mirror of `State` (src/states/mod.rs:38).  Owns one device buffer."""

    def __init__(self, num_qubits: int, dtype: int = abi.LQ_C128):
        h = C.c_void_p()
        call("lq_state_create", int(num_qubits), int(dtype), C.byref(h))
        self._h = h
        self._n = int(num_qubits)
        self._dtype = int(dtype)

    # -- lifetime --------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().lq_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- constructors (src/states/mod.rs:55-171) -------------------------
    @classmethod
    def new(cls, vector, num_qubits: int | None = None, dtype: int = abi.LQ_C128) -> "State":
        """State::new (src/states/mod.rs:55-75): validates 2^n and normalizes."""
        v = np.ascontiguousarray(np.asarray(vector, dtype=np.complex128))
        n = num_qubits if num_qubits is not None else int(math.log2(len(v))) if len(v) else 0
        if len(v) != (1 << n):
            raise LogosQError(abi.LQ_ERR_STATE_DIMENSION,
                              f"Invalid state dimension: {len(v)} (must be a power of 2)")
        s = cls(n, dtype)
        s.set_vector(v)
        s.normalize()
        return s

    @classmethod
    def new_unchecked(cls, vector, num_qubits: int) -> "State":
        s = cls(num_qubits)
        s.set_vector(np.asarray(vector, dtype=np.complex128))
        s.normalize()
        return s

    @classmethod
    def zero_state(cls, num_qubits: int, dtype: int = abi.LQ_C128) -> "State":
        return cls(num_qubits, dtype)  # created as |0...0>

    @classmethod
    def one_state(cls, num_qubits: int, dtype: int = abi.LQ_C128) -> "State":
        s = cls(num_qubits, dtype)
        call("lq_state_set_basis", s._h, C.c_uint64((1 << num_qubits) - 1))
        return s

    @classmethod
    def plus_state(cls, num_qubits: int, dtype: int = abi.LQ_C128) -> "State":
        s = cls(num_qubits, dtype)
        call("lq_state_set_plus", s._h)
        return s

    @classmethod
    def bell_state(cls) -> "State":
        s = cls(2)
        r = 1.0 / math.sqrt(2.0)
        s.set_vector(np.array([r, 0, 0, r], dtype=np.complex128))
        return s

    def clone(self) -> "State":
        s = State(self._n, self._dtype)
        call("lq_state_copy", s._h, self._h)
        return s

    # -- accessors -------------------------------------------------------
    def num_qubits(self) -> int:
        return self._n

    @property
    def dtype(self) -> int:
        return self._dtype

    def vector(self) -> np.ndarray:
        """Download the amplitudes (complex128 numpy array of length 2^n)."""
        out = np.empty(1 << self._n, dtype=np.complex128)
        call("lq_state_download", self._h, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
             C.c_size_t(1 << self._n))
        return out

    def set_vector(self, v) -> None:
        """Overwrite the amplitudes (vector_mut, src/states/mod.rs:131-133)."""
        a = np.ascontiguousarray(np.asarray(v, dtype=np.complex128))
        call("lq_state_upload", self._h, a.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
             C.c_size_t(len(a)))

    def synchronize(self) -> None:
        call("lq_state_synchronize", self._h)

    # -- numerics (src/states/mod.rs:91-365) -----------------------------
    def normalize(self) -> None:
        call("lq_normalize", self._h)

    def norm_sqr(self) -> float:
        out = C.c_double()
        call("lq_norm_sqr", self._h, C.byref(out))
        return out.value

    def probabilities(self) -> np.ndarray:
        out = np.empty(1 << self._n, dtype=np.float64)
        call("lq_probabilities", self._h, out.ctypes.data_as(C.POINTER(C.c_double)),
             C.c_size_t(len(out)))
        return out

    def probability(self, basis_state: int) -> float:
        out = C.c_double()
        call("lq_probability", self._h, C.c_uint64(int(basis_state)), C.byref(out))
        return out.value

    def inner_product_parallel(self, other: "State") -> complex:
        out = (C.c_double * 2)()
        call("lq_inner_product", self._h, other._h, out)
        return complex(out[0], out[1])

    inner_product = inner_product_parallel

    def measure_shots_parallel(self, n_shots: int, seed: int = 0) -> dict[int, int]:
        """measure_shots_parallel (src/states/mod.rs:244-258): counts per basis index."""
        out = np.empty(int(n_shots), dtype=np.uint64)
        call("lq_measure_shots", self._h, C.c_uint64(int(n_shots)), C.c_uint64(int(seed)),
             out.ctypes.data_as(C.POINTER(C.c_uint64)))
        idx, cnt = np.unique(out, return_counts=True)
        return {int(i): int(c) for i, c in zip(idx, cnt)}

    measure_shots = measure_shots_parallel

    def measure(self, seed: int = 0) -> int:
        """State::measure (src/states/mod.rs:180-185): one sampled basis index."""
        out = np.empty(1, dtype=np.uint64)
        call("lq_measure_shots", self._h, C.c_uint64(1), C.c_uint64(int(seed)),
             out.ctypes.data_as(C.POINTER(C.c_uint64)))
        return int(out[0])

    def measure_qubit(self, qubit_idx: int, seed: int = 0) -> int:
        """State::measure_qubit (src/states/mod.rs:197-238).

        The reference tests bit `qubit_idx` of the basis index (mask
        1 << qubit_idx), unlike the gates which use bit n-1-q; this mirror keeps
        that rule.  The projection and renormalisation run on the device.
        """
        if qubit_idx >= self._n or qubit_idx < 0:
            raise LogosQError(abi.LQ_ERR_QUBIT_INDEX,
                              f"Invalid qubit index: {qubit_idx} (must be < {self._n})")
        q_big_endian = self._n - 1 - qubit_idx
        term = np.zeros(1, dtype=abi.TERM_DTYPE)
        term["coefficient"] = 1.0
        term["zmask"] = np.uint64(1 << qubit_idx)
        out = C.c_double()
        call("lq_expectation_pauli", self._h, abi.term_ptr(term), 1, abi.Y_REFERENCE, C.byref(out),
             None)
        prob_one = (1.0 - out.value) / 2.0
        rng = np.random.default_rng(seed)
        result = 1 if rng.random() < prob_one else 0
        keep = [1.0, 0.0, 0.0, 0.0] if result == 0 else [0.0, 0.0, 1.0, 0.0]
        ph = np.array(keep, dtype=np.float64)
        qs = (C.c_int * 1)(q_big_endian)
        call("lq_apply_diagonal", self._h, 1, qs, ph.ctypes.data_as(C.POINTER(C.c_double)))
        self.normalize()
        return result

    def tensor_product(self, other: "State") -> "State":
        """|self> (x) |other> (src/states/mod.rs:298-314), computed on the device."""
        s = State(self._n + other._n)
        call("lq_state_tensor_product", s._h, self._h, other._h)
        return s

    def apply_gate(self, gate) -> None:
        gate.apply(self)

    # -- QuantumStateBackend (src/states/backend.rs:14-60), as State implements
    # it (src/states/mod.rs:394-486): each call applies the gate, then normalises.
    def _check_backend_qubit(self, *qubits):
        for q in qubits:
            if not 0 <= q < self._n:
                raise LogosQError(abi.LQ_ERR_QUBIT_INDEX,
                                  f"Invalid qubit index: {q} (must be < {self._n})")

    @staticmethod
    def _interleaved(matrix, dim):
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
        if m.shape != (dim, dim):
            raise LogosQError(abi.LQ_ERR_DIMENSION_MISMATCH,
                              f"Dimension mismatch: expected {dim}, got {m.shape}")
        return m.view(np.float64).reshape(-1)

    def apply_single_qubit_matrix(self, qubit: int, matrix) -> None:
        """apply_single_qubit_matrix (src/states/mod.rs:399-439): the 2x2 on one
        qubit (one device sweep), then normalise."""
        self._check_backend_qubit(qubit)
        m = self._interleaved(matrix, 2)
        call("lq_apply_matrix1", self._h, int(qubit), m.ctypes.data_as(C.POINTER(C.c_double)))
        self.normalize()

    def apply_two_qubit_matrix(self, control: int, target: int, matrix) -> None:
        """apply_two_qubit_matrix (src/states/mod.rs:441-457): the 4x4 with
        `control` as the high bit of its index (as the reference expands it),
        then normalise."""
        self._check_backend_qubit(control, target)
        m = self._interleaved(matrix, 4)
        call("lq_apply_matrix2", self._h, int(control), int(target),
             m.ctypes.data_as(C.POINTER(C.c_double)))
        self.normalize()

    def apply_three_qubit_matrix(self, q1: int, q2: int, q3: int, matrix) -> None:
        """apply_three_qubit_matrix (src/states/mod.rs:459-469): as in the
        reference, the matrix is applied to the full state (the qubit indices
        are not used)."""
        self.apply_full_matrix(matrix)

    def apply_full_matrix(self, matrix) -> None:
        """apply_full_matrix (src/states/mod.rs:471-486): the 2^n x 2^n matrix on
        the device, then normalise."""
        from .gates import MatrixGate
        MatrixGate(matrix).apply(self)

    def print(self) -> str:
        v = self.vector()
        lines = [f"State: {self._n} qubit{'s' if self._n != 1 else ''}"]
        for i, a in enumerate(v):
            p = abs(a) ** 2
            if p > 1e-10:
                lines.append(f"|{i:0{self._n}b}⟩ : {a.real:.4f}{a.imag:+.4f}i (p={p:.4f})")
        return "\n".join(lines) + "\n"

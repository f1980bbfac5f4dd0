"""Gate structs and constructors: the drop-in for src/gates/*.rs.

Each class carries the fields of the reference struct and builds one packed
`lq_gate` descriptor; `apply(state)` runs one in-place sweep on the device
(Gate::apply, src/gates/mod.rs:26-35).
"""
from __future__ import annotations

import ctypes as C
import enum
import math

import numpy as np

from . import abi
from ._lib import LogosQError, call


def make_desc(kind: int, qubits, angles=(), flags: int = 0, matrix=None,
              params=None, scales=None) -> np.ndarray:
    """One descriptor record (numpy, C layout of lq_gate)."""
    d = abi.empty_gates(1)
    d["kind"][0] = kind
    d["flags"][0] = flags
    for i, q in enumerate(qubits):
        d["q"][0, i] = int(q)
    for i, a in enumerate(angles):
        d["angle"][0, i] = float(a)
    if params is not None:
        for i, p in enumerate(params):
            d["param"][0, i] = -1 if p is None else int(p)
    if scales is not None:
        for i, s in enumerate(scales):
            d["scale"][0, i] = float(s)
    if matrix is not None:
        m = np.asarray(matrix, dtype=np.complex128).reshape(-1)
        d["m"][0, : 2 * len(m)] = m.view(np.float64)
    return d


# ---- src/gates/utils.rs: qubit q is bit n-1-q of the basis index ----------
def qubit_bit_position(qubit: int, num_qubits: int) -> int:
    return num_qubits - 1 - qubit


def qubit_mask(qubit: int, num_qubits: int) -> int:
    return 1 << qubit_bit_position(qubit, num_qubits)


def is_qubit_set(basis_index: int, qubit: int, num_qubits: int) -> bool:
    return (basis_index & qubit_mask(qubit, num_qubits)) != 0


def flip_qubit(basis_index: int, qubit: int, num_qubits: int) -> int:
    return basis_index ^ qubit_mask(qubit, num_qubits)


class RotationAxis(enum.Enum):
    """RotationAxis (src/gates/parameterized.rs:15-21)."""
    X = 0
    Y = 1
    Z = 2


class Gate:
    """Trait `Gate` (src/gates/mod.rs:26-35)."""

    @classmethod
    def new(cls, *args):
        """The gate structs' ::new constructors (same arguments as the class)."""
        return cls(*args)

    def descriptor(self) -> np.ndarray:  # pragma: no cover - abstract
        raise NotImplementedError

    def apply(self, state) -> None:
        d = self.descriptor()
        n = getattr(self, "num_qubits", None)
        if n is not None and n != state.num_qubits() and self._checks_qubits:
            raise LogosQError(abi.LQ_ERR_QUBIT_MISMATCH,
                              f"State qubit count mismatch: gate built for {n}, "
                              f"state has {state.num_qubits()}")
        call("lq_apply_gate", state.handle, abi.gate_ptr(d), None, 0)

    # The parameterized structs assert the qubit count (parameterized.rs:51);
    # the fixed structs do not.
    _checks_qubits = False


class _OneQubit(Gate):
    KIND = -1

    def __init__(self, qubit: int, num_qubits: int):
        self.qubit = qubit
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(self.KIND, [self.qubit])


class XGate(_OneQubit):
    KIND = abi.X


class YGate(_OneQubit):
    """src/gates/single_qubit.rs:39-58 (applies -Y, as the reference struct does)."""
    KIND = abi.Y


class ZGate(_OneQubit):
    KIND = abi.Z


class HGate(_OneQubit):
    KIND = abi.H


class SGate(_OneQubit):
    KIND = abi.S


class TGate(_OneQubit):
    KIND = abi.T


class _Rot1(Gate):
    KIND = -1
    _checks_qubits = True

    def __init__(self, qubit: int, theta: float, num_qubits: int):
        self.qubit = qubit
        self.theta = theta
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(self.KIND, [self.qubit], [self.theta])


class RXGate(_Rot1):
    KIND = abi.RX


class RYGate(_Rot1):
    KIND = abi.RY


class RZGate(_Rot1):
    KIND = abi.RZ


class PhaseGate(_Rot1):
    KIND = abi.PHASE


class U3Gate(Gate):
    _checks_qubits = True

    def __init__(self, qubit: int, theta: float, phi: float, lambda_: float, num_qubits: int):
        self.qubit, self.theta, self.phi, self.lambda_ = qubit, theta, phi, lambda_
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(abi.U3, [self.qubit], [self.theta, self.phi, self.lambda_])


class _Two(Gate):
    KIND = -1

    def __init__(self, a: int, b: int, num_qubits: int):
        self.a, self.b = a, b
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(self.KIND, [self.a, self.b])


class CNOTGate(_Two):
    KIND = abi.CNOT

    @property
    def control(self):
        return self.a

    @property
    def target(self):
        return self.b


class SWAPGate(_Two):
    KIND = abi.SWAP


class CZGate(_Two):
    KIND = abi.CZ


class CPhaseGate(Gate):
    """src/gates/two_qubit.rs:100-134."""

    def __init__(self, control: int, target: int, angle: float, num_qubits: int):
        self.control, self.target, self.angle = control, target, angle
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(abi.CPHASE, [self.control, self.target], [self.angle])


class ToffoliGate(Gate):
    def __init__(self, control1: int, control2: int, target: int, num_qubits: int):
        self.control1, self.control2, self.target = control1, control2, target
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(abi.TOFFOLI, [self.control1, self.control2, self.target])


class _CRot(Gate):
    KIND = -1
    _checks_qubits = True

    def __init__(self, control: int, target: int, theta: float, num_qubits: int):
        self.control, self.target, self.theta = control, target, theta
        self.num_qubits = num_qubits

    def descriptor(self):
        return make_desc(self.KIND, [self.control, self.target], [self.theta])


class CRXGate(_CRot):
    KIND = abi.CRX


class CRYGate(_CRot):
    KIND = abi.CRY


class CRZGate(_CRot):
    KIND = abi.CRZ


class CPhaseParamGate(_CRot):
    KIND = abi.CPHASE_PARAM


class _RPP(Gate):
    KIND = -1
    _checks_qubits = True

    def __init__(self, qubit1: int, qubit2: int, theta: float, num_qubits: int,
                 textbook: bool = False):
        self.qubit1, self.qubit2, self.theta = qubit1, qubit2, theta
        self.num_qubits = num_qubits
        self.textbook = textbook

    def descriptor(self):
        return make_desc(self.KIND, [self.qubit1, self.qubit2], [self.theta],
                         flags=abi.FLAG_TEXTBOOK if self.textbook else 0)


class RXXGate(_RPP):
    """src/gates/parameterized.rs:528-580.  By default the reference's loop rule
    is kept: the |01>,|10> block is skipped when qubit1 < qubit2.  Pass
    textbook=True for the full exp(-i theta XX / 2)."""
    KIND = abi.RXX


class RYYGate(_RPP):
    KIND = abi.RYY


class RZZGate(_RPP):
    KIND = abi.RZZ


class MatrixGate(Gate):
    """Generic matrix gate (src/gates/mod.rs:56-93).

    Like the reference, the matrix acts on the FULL state (2^n x 2^n) and the
    state is renormalised afterwards.  It is applied by a dense device kernel
    (O(4^n), n <= 13).
    """

    def __init__(self, matrix):
        self.matrix = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))

    def apply(self, state) -> None:
        dim = self.matrix.shape[1]
        if dim != (1 << state.num_qubits()):
            raise LogosQError(abi.LQ_ERR_DIMENSION_MISMATCH,
                              f"Matrix columns ({dim}) must match state dimension "
                              f"({1 << state.num_qubits()})")
        m = self.matrix.view(np.float64).reshape(-1)
        call("lq_apply_dense", state.handle, m.ctypes.data_as(C.POINTER(C.c_double)),
             C.c_uint64(dim))


# ---- constructors (names of src/gates/*.rs) -----------------------------
def x(qubit, num_qubits): return XGate(qubit, num_qubits)
def y(qubit, num_qubits): return YGate(qubit, num_qubits)
def z(qubit, num_qubits): return ZGate(qubit, num_qubits)
def h(qubit, num_qubits): return HGate(qubit, num_qubits)
def s(qubit, num_qubits): return SGate(qubit, num_qubits)
def t(qubit, num_qubits): return TGate(qubit, num_qubits)
def cnot(control, target, num_qubits): return CNOTGate(control, target, num_qubits)
def swap(qubit1, qubit2, num_qubits): return SWAPGate(qubit1, qubit2, num_qubits)
def cz(control, target, num_qubits): return CZGate(control, target, num_qubits)
def cphase(control, target, angle, num_qubits): return CPhaseGate(control, target, angle, num_qubits)
def toffoli(c1, c2, target, num_qubits): return ToffoliGate(c1, c2, target, num_qubits)
def rx(qubit, theta, num_qubits): return RXGate(qubit, theta, num_qubits)
def ry(qubit, theta, num_qubits): return RYGate(qubit, theta, num_qubits)
def rz(qubit, theta, num_qubits): return RZGate(qubit, theta, num_qubits)
def phase(qubit, theta, num_qubits): return PhaseGate(qubit, theta, num_qubits)
def u3(qubit, theta, phi, lambda_, num_qubits): return U3Gate(qubit, theta, phi, lambda_, num_qubits)
def crx(control, target, theta, num_qubits): return CRXGate(control, target, theta, num_qubits)
def cry(control, target, theta, num_qubits): return CRYGate(control, target, theta, num_qubits)
def crz(control, target, theta, num_qubits): return CRZGate(control, target, theta, num_qubits)
def cphase_param(control, target, theta, num_qubits):
    return CPhaseParamGate(control, target, theta, num_qubits)
def rxx(q1, q2, theta, num_qubits): return RXXGate(q1, q2, theta, num_qubits)
def ryy(q1, q2, theta, num_qubits): return RYYGate(q1, q2, theta, num_qubits)
def rzz(q1, q2, theta, num_qubits): return RZZGate(q1, q2, theta, num_qubits)


# ---- 2x2 / 4x4 matrices of src/gates/matrix.rs ----------------------------
_R2 = 1.0 / math.sqrt(2.0)


def x_matrix():
    return np.array([[0, 1], [1, 0]], dtype=np.complex128)


def y_matrix():
    return np.array([[0, -1j], [1j, 0]], dtype=np.complex128)


def z_matrix():
    return np.array([[1, 0], [0, -1]], dtype=np.complex128)


def h_matrix():
    return np.array([[_R2, _R2], [_R2, -_R2]], dtype=np.complex128)


def s_matrix():
    return np.array([[1, 0], [0, 1j]], dtype=np.complex128)


def t_matrix():
    return np.array([[1, 0], [0, complex(_R2, _R2)]], dtype=np.complex128)


def rx_matrix(theta):
    c, s_ = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return np.array([[c, -1j * s_], [-1j * s_, c]], dtype=np.complex128)


def ry_matrix(theta):
    c, s_ = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return np.array([[c, -s_], [s_, c]], dtype=np.complex128)


def rz_matrix(theta):
    c, s_ = math.cos(theta / 2.0), math.sin(theta / 2.0)
    return np.array([[complex(c, -s_), 0], [0, complex(c, s_)]], dtype=np.complex128)


def cnot_matrix():
    m = np.eye(4, dtype=np.complex128)
    m[[2, 3]] = m[[3, 2]]
    return m


def swap_matrix():
    m = np.eye(4, dtype=np.complex128)
    m[[1, 2]] = m[[2, 1]]
    return m


def cz_matrix():
    return np.diag([1, 1, 1, -1]).astype(np.complex128)


def toffoli_matrix():
    m = np.eye(8, dtype=np.complex128)
    m[[6, 7]] = m[[7, 6]]
    return m


# ---- gates::matrix constructors (src/gates/matrix.rs:14-261): MatrixGate ----
def x_gate(): return MatrixGate(x_matrix())
def y_gate(): return MatrixGate(y_matrix())
def z_gate(): return MatrixGate(z_matrix())
def h_gate(): return MatrixGate(h_matrix())
def s_gate(): return MatrixGate(s_matrix())
def t_gate(): return MatrixGate(t_matrix())
def rx_gate(theta): return MatrixGate(rx_matrix(theta))
def ry_gate(theta): return MatrixGate(ry_matrix(theta))
def rz_gate(theta): return MatrixGate(rz_matrix(theta))
def cnot_gate(): return MatrixGate(cnot_matrix())
def swap_gate(): return MatrixGate(swap_matrix())
def cz_gate(): return MatrixGate(cz_matrix())
def toffoli_gate(): return MatrixGate(toffoli_matrix())

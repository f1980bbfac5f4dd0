"""ctypes mirror of include/logosq_b200.h (types and constants only, no library load).

Kept import-light so the oracle wrapper and CPU-only tests can use the same
descriptor layout without a GPU or the built library.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# Status codes (mirror LogosQError, src/error.rs:9-61).
LQ_OK = 0
LQ_ERR_QUBIT_INDEX = 1
LQ_ERR_STATE_DIMENSION = 2
LQ_ERR_DIMENSION_MISMATCH = 3
LQ_ERR_GATE_MATRIX = 4
LQ_ERR_PARAM_COUNT = 5
LQ_ERR_QUBIT_MISMATCH = 6
LQ_ERR_INVALID_ARG = 7
LQ_ERR_OOM = 8
LQ_ERR_CUDA = 9
LQ_ERR_TIMEOUT = 10
LQ_ERR_UNSUPPORTED = 11

STATUS_NAMES = {
    0: "Ok", 1: "InvalidQubitIndex", 2: "InvalidStateDimension", 3: "DimensionMismatch",
    4: "InvalidGateMatrix", 5: "ParameterCountMismatch", 6: "CircuitQubitMismatch",
    7: "InvalidArgument", 8: "OutOfMemory", 9: "CudaError", 10: "Timeout", 11: "Unsupported",
}

LQ_C128 = 0
LQ_C64 = 1

# Gate kinds.
H, X, Y, Z, S, T = 0, 1, 2, 3, 4, 5
RX, RY, RZ, PHASE, U3 = 6, 7, 8, 9, 10
CNOT, SWAP, CZ, CPHASE, TOFFOLI = 11, 12, 13, 14, 15
CRX, CRY, CRZ, CPHASE_PARAM = 16, 17, 18, 19
RXX, RYY, RZZ = 20, 21, 22
MATRIX1, MATRIX2 = 23, 24

FLAG_RENORM = 1
FLAG_TEXTBOOK = 2

Y_REFERENCE = 0
Y_TEXTBOOK = 1

EXEC_FUSED = 0
EXEC_PER_GATE = 1


class LqGate(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("flags", C.c_int32),
        ("q", C.c_int32 * 3),
        ("param", C.c_int32 * 3),
        ("angle", C.c_double * 3),
        ("scale", C.c_double * 3),
        ("m", C.c_double * 32),
    ]


class LqPauliTerm(C.Structure):
    _fields_ = [
        ("coefficient", C.c_double),
        ("xmask", C.c_uint64),
        ("zmask", C.c_uint64),
        ("ny", C.c_int32),
        ("reserved", C.c_int32),
    ]


class LqVqeInstance(C.Structure):
    _fields_ = [
        ("num_qubits", C.c_int32),
        ("nops", C.c_int32),
        ("ops", C.POINTER(LqGate)),
        ("nparams", C.c_int32),
        ("nterms", C.c_int32),
        ("terms", C.POINTER(LqPauliTerm)),
    ]


# numpy views with the exact C layout, for building large gate lists quickly.
GATE_DTYPE = np.dtype(
    [
        ("kind", np.int32),
        ("flags", np.int32),
        ("q", np.int32, 3),
        ("param", np.int32, 3),
        ("angle", np.float64, 3),
        ("scale", np.float64, 3),
        ("m", np.float64, 32),
    ],
    align=True,
)
assert GATE_DTYPE.itemsize == C.sizeof(LqGate), (GATE_DTYPE.itemsize, C.sizeof(LqGate))

TERM_DTYPE = np.dtype(
    [
        ("coefficient", np.float64),
        ("xmask", np.uint64),
        ("zmask", np.uint64),
        ("ny", np.int32),
        ("reserved", np.int32),
    ],
    align=True,
)
assert TERM_DTYPE.itemsize == C.sizeof(LqPauliTerm)


def empty_gates(count: int) -> np.ndarray:
    """A zeroed gate array with unused qubit / param slots set to -1."""
    g = np.zeros(count, dtype=GATE_DTYPE)
    g["q"] = -1
    g["param"] = -1
    g["scale"] = 1.0
    return g


def gate_ptr(arr: np.ndarray):
    assert arr.dtype == GATE_DTYPE and arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(LqGate))


def term_ptr(arr: np.ndarray):
    assert arr.dtype == TERM_DTYPE and arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(LqPauliTerm))


def f64_ptr(arr: np.ndarray):
    assert arr.dtype == np.float64 and arr.flags["C_CONTIGUOUS"]
    return arr.ctypes.data_as(C.POINTER(C.c_double))

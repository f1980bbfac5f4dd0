"""logosq_b200: B200-native dense state-vector engine for LogosQ.

Python mirror of the reference API for the dense path (`State`, gates,
`Circuit`, observables, ansatz, gradient methods, optimizers, VQE) over the
C ABI of liblogosq_b200.so (include/logosq_b200.h).  All computation runs in
hand-written sm_100a kernels; there is no CPU fallback.
"""
from . import abi
from ._lib import LogosQError, device_count, lib
from .states import State
from .gates import (Gate, MatrixGate, XGate, YGate, ZGate, HGate, SGate, TGate, RXGate, RYGate,
                    RZGate, PhaseGate, U3Gate, CNOTGate, SWAPGate, CZGate, CPhaseGate,
                    ToffoliGate, CRXGate, CRYGate, CRZGate, CPhaseParamGate, RXXGate, RYYGate,
                    RZZGate)
from . import gates
from .circuits import Circuit, Operation
from .optimization import (Pauli, PauliTerm, PauliObservable, Observable, Ansatz,
                           HardwareEfficientAnsatz, RealAmplitudesAnsatz, EfficientSU2Ansatz,
                           ParameterizedCircuit, EntanglingGate, EntanglingPattern,
                           ParameterShift, FiniteDifference, GradientDescent, Adam, LBFGSB,
                           OptimizerResult, VQE, QuantumNaturalGradient)
from .algorithms import qft, rqc, xyz_heisenberg
from .qml import DressedVQC, VariationalQuantumCircuit, VQCBuilder, VQCType

__all__ = [
    "abi", "LogosQError", "device_count", "lib", "State", "Gate", "MatrixGate", "gates", "Circuit",
    "Operation", "Pauli", "PauliTerm", "PauliObservable", "Observable", "Ansatz",
    "HardwareEfficientAnsatz", "RealAmplitudesAnsatz", "EfficientSU2Ansatz",
    "ParameterizedCircuit", "EntanglingGate", "EntanglingPattern", "ParameterShift",
    "FiniteDifference", "GradientDescent", "Adam", "LBFGSB", "OptimizerResult", "VQE",
    "QuantumNaturalGradient",
    "qft", "rqc", "xyz_heisenberg",
    "VariationalQuantumCircuit", "VQCType", "VQCBuilder", "DressedVQC",
]

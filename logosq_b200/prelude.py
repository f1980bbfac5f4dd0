"""The reference's prelude (src/prelude.rs) for this package:
``from logosq_b200.prelude import *`` brings in the same names on the dense
path -- states, gates (structs, constructors, gates::matrix, utilities),
circuits, optimization, noise models and the VQC.  Not here: the MPS backend,
QLSTM and the data encoders, which this package does not provide."""
import math

from . import circuits, gates, states
from ._lib import LogosQError
from .circuits import Circuit
from .gates import (CNOTGate, CPhaseGate, CPhaseParamGate, CRXGate, CRYGate, CRZGate, CZGate,
                    Gate, HGate, MatrixGate, PhaseGate, RotationAxis, RXGate, RXXGate, RYGate,
                    RYYGate, RZGate, RZZGate, SGate, SWAPGate, TGate, ToffoliGate, U3Gate, XGate,
                    YGate, ZGate, cnot, cnot_gate, cphase, cz, cz_gate, flip_qubit, h, h_gate,
                    is_qubit_set, qubit_bit_position, qubit_mask, rx_gate, ry_gate, rz_gate, s,
                    s_gate, swap, swap_gate, t, t_gate, toffoli, toffoli_gate, x, x_gate, y,
                    y_gate, z, z_gate)
from .noise import (AmplitudeDampingNoise, CompositeNoise, DepolarizingNoise, NoiseModel,
                    NoiseParams, PhaseDampingNoise, ThermalRelaxationNoise)
from .optimization import (Adam, Ansatz, AnsatzType, FiniteDifference, GradientDescent,
                           GradientMethod, HardwareEfficientAnsatz, Observable, Optimizer,
                           OptimizerResult, ParameterizedCircuit, ParameterShift,
                           PauliObservable, PauliTerm, QuantumNaturalGradient, VQE, VQEResult)
from .qml import DressedVQC, VariationalQuantumCircuit, VQCBuilder, VQCType
from .states import QuantumStateBackend, State

FRAC_1_SQRT_2 = 1.0 / math.sqrt(2.0)
PI = math.pi
SQRT_2 = math.sqrt(2.0)

__all__ = [n for n in dir() if not n.startswith("_") and n != "math"]

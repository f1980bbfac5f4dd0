"""CPU: logosq_b200.prelude exports every name of the reference's prelude
(src/prelude.rs) on the dense path (not the MPS backend, QLSTM or data
encoders), State and the optimizers satisfy the reference's traits, and the
constants match."""
import math

import logosq_b200.prelude as P

REFERENCE_PRELUDE = """circuits gates states Circuit LogosQError Gate MatrixGate QuantumStateBackend State
cnot_gate cz_gate h_gate rx_gate ry_gate rz_gate s_gate swap_gate t_gate toffoli_gate x_gate
y_gate z_gate h s t x y z HGate SGate TGate XGate YGate ZGate cnot cphase cz swap CNOTGate
CPhaseGate CZGate SWAPGate toffoli ToffoliGate CPhaseParamGate CRXGate CRYGate CRZGate PhaseGate
RXGate RXXGate RYGate RYYGate RZGate RZZGate RotationAxis U3Gate flip_qubit is_qubit_set
qubit_bit_position qubit_mask FiniteDifference GradientMethod ParameterShift Observable
PauliObservable PauliTerm Adam GradientDescent Optimizer OptimizerResult QuantumNaturalGradient
VQEResult VQE Ansatz AnsatzType HardwareEfficientAnsatz ParameterizedCircuit
AmplitudeDampingNoise CompositeNoise DepolarizingNoise NoiseModel NoiseParams PhaseDampingNoise
ThermalRelaxationNoise DressedVQC VQCBuilder VQCType VariationalQuantumCircuit FRAC_1_SQRT_2 PI
SQRT_2""".split()


def test_every_dense_path_name_is_exported():
    missing = [n for n in REFERENCE_PRELUDE if n not in P.__all__]
    assert not missing, missing


def test_traits_and_constants():
    st = P.State.__new__(P.State)  # no device state: only the interface is checked
    assert isinstance(st, P.QuantumStateBackend)
    assert isinstance(P.GradientDescent(0.1, 10), P.Optimizer)
    assert isinstance(P.Adam(0.1, 10), P.Optimizer)
    assert P.PI == math.pi and abs(P.SQRT_2 * P.FRAC_1_SQRT_2 - 1.0) < 1e-15

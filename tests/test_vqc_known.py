"""CPU: the reference's VQC unit tests that need no simulation (src/qml/vqc.rs,
its tests module: creation, the builder, parameter counts) and DressedVQC's
post-processing (src/qml/vqc.rs:251-284) with the VQC's outputs stubbed."""
from logosq_b200 import DressedVQC, VariationalQuantumCircuit, VQCBuilder, VQCType


def test_vqc_creation():
    v = VariationalQuantumCircuit.new(4, 2)
    assert v.num_qubits() == 4 and v.num_layers == 2
    assert v.vqc_type is VQCType.BasicEntangling and v.include_input_encoding


def test_vqc_builder():
    v = VQCBuilder.new(3).with_layers(2).with_type(VQCType.StronglyEntangling).build()
    assert v.num_qubits() == 3 and v.num_layers == 2 and v.vqc_type is VQCType.StronglyEntangling
    d = VQCBuilder.new(5).build()
    assert d.num_layers == 1 and d.vqc_type is VQCType.BasicEntangling and d.include_input_encoding
    assert not VQCBuilder.new(2).with_input_encoding(False).build().include_input_encoding


def test_num_variational_params():
    assert VariationalQuantumCircuit(3, 2, VQCType.Simple).num_variational_params() == 6
    assert VariationalQuantumCircuit(3, 2, VQCType.StronglyEntangling).num_variational_params() == 18
    assert VariationalQuantumCircuit(3, 2, VQCType.BasicEntangling).num_variational_params() == 12


def test_dressed_vqc(monkeypatch):
    v = VariationalQuantumCircuit.new(2, 1)
    d = DressedVQC(v, 2)
    assert d.num_params() == v.num_variational_params() + 4
    monkeypatch.setattr(VariationalQuantumCircuit, "forward", lambda self, x, p: [0.25, -0.5])
    d.output_weights = [2.0, 3.0]
    d.output_biases = [0.1, -0.2]
    assert d.forward([0.5, 0.3], [0.1] * 4) == [0.25 * 2.0 + 0.1, -0.5 * 3.0 - 0.2]

"""CPU: the reference's gate utilities (src/gates/utils.rs: qubit q is bit
n-1-q), RotationAxis, AnsatzType, and the ::new constructors of the gate
structs, MatrixGate and the noise models, which build the same objects as the
classes."""
import numpy as np

from logosq_b200 import gates, noise
from logosq_b200.gates import (MatrixGate, RotationAxis, RXGate, flip_qubit, is_qubit_set,
                               qubit_bit_position, qubit_mask)
from logosq_b200.optimization import AnsatzType


def test_bit_conventions():
    assert qubit_bit_position(0, 3) == 2 and qubit_bit_position(2, 3) == 0
    assert qubit_mask(0, 3) == 0b100 and qubit_mask(2, 3) == 0b001
    assert is_qubit_set(0b100, 0, 3) and not is_qubit_set(0b100, 2, 3)
    assert flip_qubit(0b000, 1, 3) == 0b010 and flip_qubit(0b010, 1, 3) == 0


def test_enums():
    assert [a.name for a in RotationAxis] == ["X", "Y", "Z"]
    assert [a.name for a in AnsatzType] == ["HardwareEfficient", "RealAmplitudes",
                                            "EfficientSU2", "Custom"]


def test_new_constructors_build_the_same_objects():
    a, b = RXGate.new(1, 0.3, 3), RXGate(1, 0.3, 3)
    assert np.array_equal(a.descriptor(), b.descriptor())
    m = MatrixGate.new(gates.x_matrix())
    assert np.array_equal(m.matrix, gates.x_matrix())
    d = noise.DepolarizingNoise.new(0.1)
    assert type(d) is noise.DepolarizingNoise

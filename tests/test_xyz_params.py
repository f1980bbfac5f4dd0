"""CPU: HeisenbergParameters (src/algorithms/xyz_heisenberg.rs:8-28) and the
params forms of create_circuit: defaults, and the same Trotter circuit as the
explicit-coupling form."""
import numpy as np

from logosq_b200 import xyz_heisenberg
from logosq_b200.algorithms import HeisenbergParameters


def test_defaults():
    p = HeisenbergParameters()
    assert (p.jx, p.jy, p.jz, p.external_field, p.time_steps, p.dt) == (1.0, 1.0, 1.0, 0.0, 100,
                                                                          0.01)


def test_params_form_matches_explicit_form():
    p = HeisenbergParameters(jx=0.7, jy=-0.3, jz=1.1, external_field=0.2, time_steps=3, dt=0.05)
    a = xyz_heisenberg.create_circuit(4, p)
    b = xyz_heisenberg.create_circuit(4, 0.7, -0.3, 1.1, 0.2, 3, 0.05)
    assert a.name() == "XYZ-Heisenberg Model"
    assert np.array_equal(a.packed(), b.packed())
    # per step: 3 bond rotations on 3 bonds + 4 field rotations
    assert len(a.operations()) == 3 * (3 * 3 + 4)


def test_no_field_rotations_without_field():
    c = xyz_heisenberg.create_circuit(3, HeisenbergParameters(time_steps=2))
    assert len(c.operations()) == 2 * 3 * 2

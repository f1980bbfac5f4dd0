"""GPU: xyz_heisenberg.simulate and the params form of calculate_energy_efficient
(src/algorithms/xyz_heisenberg.rs:62-66, 143-252) against the oracle."""
import numpy as np
import pytest

import oracle
from helpers import oracle_run
from logosq_b200 import State, xyz_heisenberg
from logosq_b200.algorithms import HeisenbergParameters

pytestmark = pytest.mark.gpu


def test_simulate_and_energy_match_oracle():
    p = HeisenbergParameters(jx=0.8, jy=0.5, jz=-0.6, external_field=0.3, time_steps=5, dt=0.1)
    n = 6
    st = State.plus_state(n)
    xyz_heisenberg.simulate(st, p)
    v0 = np.full(1 << n, 1 / np.sqrt(1 << n), dtype=np.complex128)
    want = oracle_run(xyz_heisenberg.create_circuit(n, p), v0)
    assert np.abs(st.vector() - want).max() < 1e-12
    e = xyz_heisenberg.calculate_energy_efficient(st, p)
    e_want = oracle.heisenberg_energy(want, p.jx, p.jy, p.jz, p.external_field)
    assert abs(e - e_want) < 1e-12 * max(1.0, abs(e_want))

"""CPU: the noise-model oracle (numpy restatement of src/noise/mod.rs) on cases
worked out by hand from the reference's loops, and the host-side parts of the
noise mirror (thermal-relaxation rates, seeded depolarizing draws)."""
import math

import numpy as np

import oracle
from logosq_b200 import noise


def basis(n, i):
    v = np.zeros(1 << n, dtype=np.complex128)
    v[i] = 1.0
    return v


def test_pauli_errors_use_bit_qubit_and_minus_y():
    v = basis(3, 0)
    assert np.allclose(oracle.noise_pauli(v, 0, 1), basis(3, 1))   # X on bit 0
    assert np.allclose(oracle.noise_pauli(v, 2, 1), basis(3, 4))   # X on bit 2
    # Y error: new[bit set] = -i psi[bit clear]  (the reference's -Y)
    assert np.allclose(oracle.noise_pauli(v, 1, 2), -1j * basis(3, 2))
    assert np.allclose(oracle.noise_pauli(basis(3, 2), 1, 2), 1j * basis(3, 0))
    assert np.allclose(oracle.noise_pauli(basis(3, 2), 1, 3), -basis(3, 2))


def test_amplitude_damping_is_a_coherent_sum_then_normalised():
    g = 0.36
    out = oracle.noise_amplitude_damping(basis(1, 1), g, [0])
    assert np.allclose(out, [math.sqrt(g), math.sqrt(1 - g)])
    # two targets accumulate into one vector: |00> gets psi from both -> 2|00>, normalised
    assert np.allclose(oracle.noise_amplitude_damping(basis(2, 0), g, [0, 1]), basis(2, 0))
    # |11> with targets 0, 1: (sqrt(1-g)|11> + sqrt(g)|10>) + (sqrt(1-g)|11> + sqrt(g)|01>)
    want = np.array([0, math.sqrt(g), math.sqrt(g), 2 * math.sqrt(1 - g)], dtype=complex)
    want /= np.linalg.norm(want)
    assert np.allclose(oracle.noise_amplitude_damping(basis(2, 3), g, [0, 1]), want)


def test_phase_damping_keeps_only_the_last_target():
    v = np.full(4, 0.5, dtype=complex)
    lam = 0.75
    out = oracle.noise_phase_damping(v, lam, [0, 1])
    want = np.array([0.5, 0.5, 0.5 * math.sqrt(1 - lam), 0.5 * math.sqrt(1 - lam)])
    assert np.allclose(out, want / np.linalg.norm(want))


def test_thermal_relaxation_rates():
    m = noise.ThermalRelaxationNoise(t1=50.0, t2=70.0, gate_time=0.1)
    pa, pp = m.probabilities()
    assert math.isclose(pa, 1 - math.exp(-0.1 / 50.0))
    assert math.isclose(pp, 1 - math.exp(-0.1 * (1 / 70.0 - 1 / 100.0)))
    capped = noise.ThermalRelaxationNoise(t1=10.0, t2=50.0, gate_time=1.0)
    assert capped.t2 == 20.0 and capped.probabilities()[1] == 0.0


def test_depolarizing_draws_are_seeded():
    a = noise.DepolarizingNoise(0.5, seed=3).with_target_qubits([0, 2, 4])
    b = noise.DepolarizingNoise(0.5, seed=3).with_target_qubits([0, 2, 4])
    assert [a.draw(5) for _ in range(20)] == [b.draw(5) for _ in range(20)]
    assert noise.DepolarizingNoise(0.0).draw(6) == []
    full = noise.DepolarizingNoise(1.0, seed=1).draw(6)
    assert [q for q, _ in full] == list(range(6)) and all(k in (1, 2, 3) for _, k in full)
    assert "Composite(Depolarizing(p=0.5)" in noise.CompositeNoise().add_noise(a).name()

"""Noise models (mirror of src/noise/mod.rs) on the device.

As in the reference, a noise model's qubit index is the basis-index bit
(1 << qubit), not the gate convention (bit n-1-q), and every model acts on the
whole state vector:

* DepolarizingNoise (src/noise/mod.rs:60-83): per target qubit, with
  probability p, one of X, Y (the reference's -Y) or Z.  The reference draws
  from `rand::thread_rng()`, which cannot be reproduced; this mirror draws from
  a seeded SplitMix64 stream (`seed`), one uniform for the event and one for the
  Pauli per target qubit, in target order.
* AmplitudeDampingNoise (src/noise/mod.rs:108-146): sum over target qubits of
  (K0 + K1) psi, then normalised.
* PhaseDampingNoise (src/noise/mod.rs:173-210): the last target qubit's |1>
  amplitudes scaled by sqrt(1 - lambda), then normalised.
* ThermalRelaxationNoise (src/noise/mod.rs:251-292): amplitude damping with
  1 - exp(-t/T1), then phase damping with 1 - exp(-t/T_phi),
  1/T_phi = 1/T2 - 1/(2 T1), T2 capped at 2 T1.
* CompositeNoise (src/noise/mod.rs:319-328): the models in order.
"""
from __future__ import annotations

import ctypes as C
import math

from ._lib import call
from .workloads import SplitMix64


def _targets(qubits):
    if qubits is None:
        return None, 0
    arr = (C.c_int * len(qubits))(*[int(q) for q in qubits])
    return arr, len(qubits)


class NoiseModel:
    """Trait NoiseModel (src/noise/mod.rs:10-16)."""

    @classmethod
    def new(cls, *args):
        """The models' ::new constructors (same arguments as the class)."""
        return cls(*args)

    def apply(self, state) -> None:
        raise NotImplementedError

    def name(self) -> str:
        raise NotImplementedError


class NoiseParams:
    """NoiseParams (src/noise/mod.rs:19-40)."""

    def __init__(self, error_probability: float, target_qubits=None):
        self.error_probability = float(error_probability)
        self.target_qubits = None if target_qubits is None else list(target_qubits)


class DepolarizingNoise(NoiseModel):
    def __init__(self, error_probability: float, seed: int = 0):
        self.params = NoiseParams(error_probability)
        self._rng = SplitMix64(seed)

    def with_target_qubits(self, qubits) -> "DepolarizingNoise":
        self.params.target_qubits = list(qubits)
        return self

    def draw(self, num_qubits: int):
        """The (qubit, pauli) errors of one application, pauli 1 = X, 2 = Y, 3 = Z."""
        tq = self.params.target_qubits
        tq = list(range(num_qubits)) if tq is None else tq
        out = []
        for q in tq:
            hit = self._rng.uniform() < self.params.error_probability
            kind = 1 + min(int(self._rng.uniform() * 3), 2)
            if hit:
                out.append((q, kind))
        return out

    def apply(self, state) -> None:
        for q, kind in self.draw(state.num_qubits()):
            call("lq_noise_pauli", state.handle, q, kind)

    def name(self) -> str:
        return f"Depolarizing(p={self.params.error_probability})"


class AmplitudeDampingNoise(NoiseModel):
    def __init__(self, error_probability: float):
        self.params = NoiseParams(error_probability)

    def with_target_qubits(self, qubits) -> "AmplitudeDampingNoise":
        self.params.target_qubits = list(qubits)
        return self

    def apply(self, state) -> None:
        arr, nq = _targets(self.params.target_qubits)
        call("lq_noise_amplitude_damping", state.handle, self.params.error_probability, arr, nq)

    def name(self) -> str:
        return f"AmplitudeDamping(p={self.params.error_probability})"


class PhaseDampingNoise(NoiseModel):
    def __init__(self, error_probability: float):
        self.params = NoiseParams(error_probability)

    def with_target_qubits(self, qubits) -> "PhaseDampingNoise":
        self.params.target_qubits = list(qubits)
        return self

    def apply(self, state) -> None:
        arr, nq = _targets(self.params.target_qubits)
        call("lq_noise_phase_damping", state.handle, self.params.error_probability, arr, nq)

    def name(self) -> str:
        return f"PhaseDamping(p={self.params.error_probability})"


class ThermalRelaxationNoise(NoiseModel):
    def __init__(self, t1: float, t2: float, gate_time: float):
        self.t1 = float(t1)
        self.t2 = min(float(t2), 2.0 * float(t1))
        self.gate_time = float(gate_time)
        self.target_qubits = None

    def with_target_qubits(self, qubits) -> "ThermalRelaxationNoise":
        self.target_qubits = list(qubits)
        return self

    def probabilities(self):
        p_amp = 1.0 - math.exp(-self.gate_time / self.t1)
        rate = 1.0 / self.t2 - 1.0 / (2.0 * self.t1) if self.t2 <= 2.0 * self.t1 else 0.0
        p_phase = 1.0 - math.exp(-self.gate_time * rate) if rate > 0.0 else 0.0
        return p_amp, p_phase

    def apply(self, state) -> None:
        p_amp, p_phase = self.probabilities()
        if p_amp > 0.0:
            AmplitudeDampingNoise(p_amp).with_target_qubits(
                self.target_qubits or range(state.num_qubits())).apply(state)
        if p_phase > 0.0:
            PhaseDampingNoise(p_phase).with_target_qubits(
                self.target_qubits or range(state.num_qubits())).apply(state)

    def name(self) -> str:
        return f"ThermalRelaxation(T1={self.t1}, T2={self.t2}, gate_time={self.gate_time})"


class CompositeNoise(NoiseModel):
    def __init__(self):
        self.noise_models: list[NoiseModel] = []

    def add_noise(self, model: NoiseModel) -> "CompositeNoise":
        self.noise_models.append(model)
        return self

    def apply(self, state) -> None:
        for m in self.noise_models:
            m.apply(state)

    def name(self) -> str:
        return "Composite(" + ", ".join(m.name() for m in self.noise_models) + ")"

"""Workload builders: src/algorithms/{qft,rqc,xyz_heisenberg}.rs.

These produce circuits and observables for the engine; none of them computes
on the host.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .circuits import Circuit
from .optimization import Pauli, PauliObservable, PauliTerm


class qft:  # noqa: N801 - mirrors the Rust module path algorithms::qft
    """src/algorithms/qft.rs."""

    @staticmethod
    def create_circuit(num_qubits: int, gate_structs: bool = True) -> Circuit:
        """qft::create_circuit (src/algorithms/qft.rs:10-27).

        The reference adds H through Circuit::h, a dense 2^n x 2^n MatrixGate
        (usable only for tiny n).  With gate_structs=True (default) H is the
        HGate struct (src/gates/single_qubit.rs:90), the form the 20-qubit
        workload uses; gate_structs=False keeps the dense builder's semantics
        (2x2 sweep followed by renormalisation).
        """
        c = Circuit(num_qubits).with_name("Quantum Fourier Transform")
        for i in range(num_qubits):
            if gate_structs:
                c._push(_h_desc(i), [i], "H")
            else:
                c.h(i)
            for j in range(i + 1, num_qubits):
                c.cphase(i, j, math.pi / float(1 << (j - i)))
        for i in range(num_qubits // 2):
            c.swap(i, num_qubits - i - 1)
        return c

    @staticmethod
    def create_inverse_circuit(num_qubits: int, gate_structs: bool = True) -> Circuit:
        """qft::create_inverse_circuit (src/algorithms/qft.rs:30-47)."""
        c = Circuit(num_qubits).with_name("Inverse Quantum Fourier Transform")
        for i in range(num_qubits // 2):
            c.swap(i, num_qubits - i - 1)
        for i in reversed(range(num_qubits)):
            for j in range(i + 1, num_qubits):
                c.cphase(i, j, -math.pi / float(1 << (j - i)))
            if gate_structs:
                c._push(_h_desc(i), [i], "H")
            else:
                c.h(i)
        return c

    @staticmethod
    def apply(state) -> None:
        """qft::apply (src/algorithms/qft.rs:50-71).  The reference computes the
        transform with an inverse FFT scaled by 1/sqrt(N); the engine applies the
        equivalent gate sequence on the device (equal to the FFT form to ~1e-15)."""
        qft.create_circuit(state.num_qubits()).execute(state)

    @staticmethod
    def apply_inverse(state) -> None:
        """qft::apply_inverse (src/algorithms/qft.rs:74-93)."""
        qft.create_inverse_circuit(state.num_qubits()).execute(state)

    @staticmethod
    def controlled_phase(circuit: Circuit, control: int, target: int, angle: float) -> None:
        """qft::controlled_phase (src/algorithms/qft.rs:96-105)."""
        circuit.cphase(control, target, angle)


def _h_desc(q):
    from .gates import make_desc
    return make_desc(abi.H, [q])


class rqc:  # noqa: N801
    """src/algorithms/rqc.rs (random circuits)."""

    @staticmethod
    def generate_supremacy_circuit(num_qubits: int, depth: int, seed: int = 0) -> Circuit:
        """generate_supremacy_circuit (src/algorithms/rqc.rs:236-268), seeded:
        per layer RZ(phi) RY(theta) RZ(lambda) on every qubit, then CNOT(q, q+1)
        for q = layer % 2, step 2."""
        from .workloads import SplitMix64
        rng = SplitMix64(seed)
        c = Circuit(num_qubits).with_name(f"Supremacy Circuit (d={depth})")
        for layer in range(depth):
            for q in range(num_qubits):
                theta = rng.uniform(0.0, 2.0 * math.pi)
                phi = rng.uniform(0.0, 2.0 * math.pi)
                lam = rng.uniform(0.0, 2.0 * math.pi)
                c.rz(q, phi)
                c.ry(q, theta)
                c.rz(q, lam)
            for q in range(layer % 2, num_qubits - 1, 2):
                c.cnot(q, q + 1)
        return c


class xyz_heisenberg:  # noqa: N801
    """src/algorithms/xyz_heisenberg.rs."""

    @staticmethod
    def hamiltonian(num_qubits, jx, jy, jz, h=0.0) -> PauliObservable:
        """H = sum_b (Jx_b X_b X_b+1 + Jy_b Y Y + Jz_b Z Z) + sum_i h_i Z_i, open
        chain, the operator whose energy calculate_energy_efficient evaluates
        (src/algorithms/xyz_heisenberg.rs:143-163).  Couplings may be scalars
        (uniform) or per-bond / per-site sequences."""
        n = num_qubits
        jx = np.broadcast_to(np.asarray(jx, dtype=np.float64), (n - 1,))
        jy = np.broadcast_to(np.asarray(jy, dtype=np.float64), (n - 1,))
        jz = np.broadcast_to(np.asarray(jz, dtype=np.float64), (n - 1,))
        hh = np.broadcast_to(np.asarray(h, dtype=np.float64), (n,))
        obs = PauliObservable(n)
        for i in range(n - 1):
            for coef, p in ((jx[i], Pauli.X), (jy[i], Pauli.Y), (jz[i], Pauli.Z)):
                ps = [Pauli.I] * n
                ps[i] = p
                ps[i + 1] = p
                obs.add_term(PauliTerm(float(coef), ps))
        if np.any(hh != 0.0):
            for i in range(n):
                ps = [Pauli.I] * n
                ps[i] = Pauli.Z
                obs.add_term(PauliTerm(float(hh[i]), ps))
        return obs

    @staticmethod
    def calculate_energy_efficient(state, jx, jy, jz, external_field=0.0) -> float:
        return xyz_heisenberg.hamiltonian(state.num_qubits(), jx, jy, jz,
                                          external_field).expectation(state)

    @staticmethod
    def create_circuit(num_qubits, jx, jy, jz, external_field, time_steps, dt,
                       textbook=False) -> Circuit:
        """create_circuit (src/algorithms/xyz_heisenberg.rs:31-59): Trotter steps of
        RXX/RYY/RZZ(2*J*dt) on each bond and RZ(h*dt).  RXX/RYY keep the
        reference's loop rule unless textbook=True."""
        c = Circuit(num_qubits).with_name("XYZ-Heisenberg Model")
        for _ in range(time_steps):
            for i in range(num_qubits - 1):
                c.rxx(i, i + 1, 2.0 * jx * dt, textbook=textbook)
            for i in range(num_qubits - 1):
                c.ryy(i, i + 1, 2.0 * jy * dt, textbook=textbook)
            for i in range(num_qubits - 1):
                c.rzz(i, i + 1, 2.0 * jz * dt)
            if external_field != 0.0:
                for i in range(num_qubits):
                    c.rz(i, external_field * dt)
        return c

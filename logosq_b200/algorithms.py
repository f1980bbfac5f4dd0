"""Workload builders: src/algorithms/{qft,rqc,xyz_heisenberg}.rs.

These produce circuits and observables for the engine; none of them computes
on the host.
"""
from __future__ import annotations

import enum
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


class RandomGateType(enum.Enum):
    """RandomGateType (src/algorithms/rqc.rs:11-16)."""
    Single = 0
    TwoQubit = 1
    Rotation = 2


class RandomCircuitConfig:
    """RandomCircuitConfig and its Default (src/algorithms/rqc.rs:19-39): 3
    qubits, depth 10, gate types Single 0.5 / TwoQubit 0.3 / Rotation 0.2, no
    seed."""

    def __init__(self, num_qubits=3, depth=10, gate_types=None, seed=None):
        self.num_qubits, self.depth, self.seed = num_qubits, depth, seed
        self.gate_types = list(gate_types) if gate_types is not None else [
            (RandomGateType.Single, 0.5), (RandomGateType.TwoQubit, 0.3),
            (RandomGateType.Rotation, 0.2)]


class rqc:  # noqa: N801
    """src/algorithms/rqc.rs (random circuits).

    The generators follow the reference's construction -- per depth step one
    gate type drawn by weight, then a random qubit (pair), gate and angle, with
    CZ written as H.CNOT.H and SWAP as three CNOTs -- but draw from the
    project's SplitMix64 stream: the reference's StdRng (ChaCha12) stream
    cannot be reproduced here, so equal seeds give the same circuits within
    this package, not the reference's circuits.  No seed draws one from the
    operating system, as the reference seeds from entropy.
    """

    RandomGateType = RandomGateType
    RandomCircuitConfig = RandomCircuitConfig

    @staticmethod
    def _rng(seed):
        import os
        from .workloads import SplitMix64
        return SplitMix64(int.from_bytes(os.urandom(8), "little") if seed is None else seed)

    @staticmethod
    def _select(gate_types, rng):
        # select_gate_type (rqc.rs:80-95): weighted choice; invalid weights -> Single
        w = [p for _, p in gate_types]
        if not w or any(x < 0 or not math.isfinite(x) for x in w) or sum(w) <= 0:
            return RandomGateType.Single
        u, acc = rng.uniform() * sum(w), 0.0
        for (t, p) in gate_types:
            acc += p
            if u < acc:
                return t
        return gate_types[-1][0]

    @staticmethod
    def generate(config: RandomCircuitConfig) -> Circuit:
        """generate (src/algorithms/rqc.rs:42-77)."""
        n = config.num_qubits
        c = Circuit(n).with_name(f"Random Circuit (d={config.depth})")
        rng = rqc._rng(config.seed)
        for _ in range(config.depth):
            t = rqc._select(config.gate_types, rng)
            if t == RandomGateType.TwoQubit and n < 2:
                t = RandomGateType.Single
            if t == RandomGateType.Single:
                q = rng.randint(0, n - 1)
                (c.h, c.x, c.y, c.z, c.s, c.t)[rng.randint(0, 5)](q)
            elif t == RandomGateType.TwoQubit:
                q1 = rng.randint(0, n - 1)
                q2 = rng.randint(0, n - 1)
                while q2 == q1:
                    q2 = rng.randint(0, n - 1)
                k = rng.randint(0, 2)
                if k == 0:
                    c.cnot(q1, q2)
                elif k == 1:
                    c.h(q2)
                    c.cnot(q1, q2)
                    c.h(q2)
                else:
                    c.cnot(q1, q2)
                    c.cnot(q2, q1)
                    c.cnot(q1, q2)
            else:
                q = rng.randint(0, n - 1)
                angle = rng.uniform(0.0, 2.0 * math.pi)
                (c.rx, c.ry, c.rz)[rng.randint(0, 2)](q, angle)
        return c

    @staticmethod
    def apply(state, config: RandomCircuitConfig) -> None:
        """apply (src/algorithms/rqc.rs:185-190)."""
        rqc.generate(config).execute(state)

    @staticmethod
    def generate_simple(num_qubits: int, depth: int, seed=None) -> Circuit:
        """generate_simple (src/algorithms/rqc.rs:194-207): weights 0.4 / 0.4 / 0.2."""
        return rqc.generate(RandomCircuitConfig(
            num_qubits, depth, [(RandomGateType.Single, 0.4), (RandomGateType.TwoQubit, 0.4),
                                (RandomGateType.Rotation, 0.2)], seed))

    @staticmethod
    def generate_2design(num_qubits: int, seed=None) -> Circuit:
        """generate_2design (src/algorithms/rqc.rs:211-232): depth 2 n^2, weights
        0.3 / 0.5 / 0.2.  (The reference takes no seed; the optional one here
        makes the circuit reproducible.)"""
        depth = 2 * num_qubits * num_qubits
        c = rqc.generate(RandomCircuitConfig(
            num_qubits, depth, [(RandomGateType.Single, 0.3), (RandomGateType.TwoQubit, 0.5),
                                (RandomGateType.Rotation, 0.2)], seed))
        return c.with_name(f"2-Design Random Circuit (n={num_qubits}, d={depth})")

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


class HeisenbergParameters:
    """HeisenbergParameters and its Default (src/algorithms/xyz_heisenberg.rs:8-28)."""

    def __init__(self, jx=1.0, jy=1.0, jz=1.0, external_field=0.0, time_steps=100, dt=0.01):
        self.jx, self.jy, self.jz = jx, jy, jz
        self.external_field, self.time_steps, self.dt = external_field, time_steps, dt


class xyz_heisenberg:  # noqa: N801
    """src/algorithms/xyz_heisenberg.rs.  The reference's functions take a
    HeisenbergParameters; these accept one in place of the explicit couplings.
    (calculate_energy, the reference's slow variant, takes an unconjugated
    product Re sum_i psi_i (P psi)_i per Pauli string, which equals the
    expectation only for real amplitudes; it is not provided: use
    calculate_energy_efficient.)"""

    HeisenbergParameters = HeisenbergParameters

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
    def calculate_energy_efficient(state, jx, jy=None, jz=None, external_field=0.0) -> float:
        """calculate_energy_efficient (src/algorithms/xyz_heisenberg.rs:143-252):
        (state, params) or (state, jx, jy, jz[, external_field])."""
        if isinstance(jx, HeisenbergParameters):
            p = jx
            jx, jy, jz, external_field = p.jx, p.jy, p.jz, p.external_field
        return xyz_heisenberg.hamiltonian(state.num_qubits(), jx, jy, jz,
                                          external_field).expectation(state)

    @staticmethod
    def simulate(state, params: HeisenbergParameters) -> None:
        """simulate (src/algorithms/xyz_heisenberg.rs:62-66): the Trotter circuit
        of create_circuit executed on the state."""
        xyz_heisenberg.create_circuit(state.num_qubits(), params).execute(state)

    @staticmethod
    def create_circuit(num_qubits, jx, jy=None, jz=None, external_field=None, time_steps=None,
                       dt=None, textbook=False) -> Circuit:
        """create_circuit (src/algorithms/xyz_heisenberg.rs:31-59): Trotter steps of
        RXX/RYY/RZZ(2*J*dt) on each bond and RZ(h*dt).  RXX/RYY keep the
        reference's loop rule unless textbook=True.  Takes (num_qubits, params)
        or the explicit couplings."""
        if isinstance(jx, HeisenbergParameters):
            p = jx
            jx, jy, jz, external_field, time_steps, dt = (p.jx, p.jy, p.jz, p.external_field,
                                                          p.time_steps, p.dt)
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

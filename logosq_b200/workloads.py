"""Seeded synthetic workloads (no datasets are involved anywhere).

Random numbers come from SplitMix64 (Steele, Lea & Flood 2014): state +=
0x9E3779B97F4A7C15, then two xor-shift-multiply rounds.  Uniform doubles take
the top 53 bits; Gaussians use Box-Muller on two uniforms.  The same streams
feed the engine, the oracle and the tests, so every comparison sees identical
inputs.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

_M64 = (1 << 64) - 1
_GOLD = 0x9E3779B97F4A7C15
_C1 = 0xBF58476D1CE4E5B9
_C2 = 0x94D049BB133111EB


class SplitMix64:
    def __init__(self, seed: int):
        self.state = int(seed) & _M64

    def next_u64(self) -> int:
        self.state = (self.state + _GOLD) & _M64
        z = self.state
        z = ((z ^ (z >> 30)) * _C1) & _M64
        z = ((z ^ (z >> 27)) * _C2) & _M64
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / 9007199254740992.0))

    def randint(self, lo: int, hi_inclusive: int) -> int:
        return lo + int(self.uniform() * (hi_inclusive - lo + 1))


def splitmix_stream(seed: int, count: int) -> np.ndarray:
    """count consecutive SplitMix64 outputs as uint64 (vectorised)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(int(seed) & _M64) + k * np.uint64(_GOLD)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(_C1)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(_C2)
        return z ^ (z >> np.uint64(31))


def uniform_stream(seed: int, count: int, lo=0.0, hi=1.0) -> np.ndarray:
    u = (splitmix_stream(seed, count) >> np.uint64(11)).astype(np.float64) * (
        1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u


def gaussian_state(num_qubits: int, seed: int) -> np.ndarray:
    """i.i.d. complex Gaussian amplitudes (re, im ~ N(0,1)), normalised in FP64."""
    N = 1 << num_qubits
    u = uniform_stream(seed, 2 * N)
    u1 = np.maximum(u[0::2], 1e-300)
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    re = r * np.cos(2.0 * math.pi * u2)
    im = r * np.sin(2.0 * math.pi * u2)
    v = re + 1j * im
    v /= math.sqrt(float(np.sum(re * re + im * im)))
    return v


def qft_gates(num_qubits: int) -> np.ndarray:
    """The gate list of qft::create_circuit (src/algorithms/qft.rs:10-27) with the
    HGate struct for H: n H + n(n-1)/2 CPhase + n/2 SWAP descriptors."""
    n = num_qubits
    count = n + n * (n - 1) // 2 + n // 2
    g = abi.empty_gates(count)
    k = 0
    for i in range(n):
        g[k]["kind"] = abi.H
        g[k]["q"][0] = i
        k += 1
        for j in range(i + 1, n):
            g[k]["kind"] = abi.CPHASE
            g[k]["q"][0], g[k]["q"][1] = i, j
            g[k]["angle"][0] = math.pi / float(1 << (j - i))
            k += 1
    for i in range(n // 2):
        g[k]["kind"] = abi.SWAP
        g[k]["q"][0], g[k]["q"][1] = i, n - i - 1
        k += 1
    return g


def brickwork_u3(num_qubits: int, layers: int, seed: int) -> np.ndarray:
    """Random U3 + CNOT brickwork: per layer U3(theta, phi, lambda) on every qubit
    (angles uniform in [0, 2 pi), drawn theta, phi, lambda per qubit in order),
    then CNOT(q, q+1) for q = layer % 2, step 2 (src/algorithms/rqc.rs:258-264)."""
    n = num_qubits
    ang = uniform_stream(seed, 3 * n * layers, 0.0, 2.0 * math.pi).reshape(layers, n, 3)
    recs = []
    for layer in range(layers):
        u = abi.empty_gates(n)
        u["kind"] = abi.U3
        u["q"][:, 0] = np.arange(n)
        u["angle"][:, :] = ang[layer]
        recs.append(u)
        qs = np.arange(layer % 2, n - 1, 2)
        c = abi.empty_gates(len(qs))
        c["kind"] = abi.CNOT
        c["q"][:, 0] = qs
        c["q"][:, 1] = qs + 1
        recs.append(c)
    return np.concatenate(recs)


def brickwork_bytes(num_qubits: int, layers: int, amp_bytes: int = 16) -> int:
    """Algorithmic bytes of the brickwork: U3 reads+writes the state (2S), CNOT
    reads+writes the half it permutes (S)."""
    S = amp_bytes << num_qubits
    total = 0
    for layer in range(layers):
        ncx = len(range(layer % 2, num_qubits - 1, 2))
        total += num_qubits * 2 * S + ncx * S
    return total


def qft_bytes(num_qubits: int, amp_bytes: int = 16) -> int:
    """H: 2S ; CPhase: the |11> quarter read+written, S/2 ; SWAP: the |01>,|10>
    half read+written, S."""
    S = amp_bytes << num_qubits
    n = num_qubits
    return n * 2 * S + (n * (n - 1) // 2) * (S // 2) + (n // 2) * S


def heisenberg_instances(count: int, seed: int, n_lo=10, n_hi=20, layers=4):
    """Batching workload: XYZ open chains with per-bond Jx, Jy, Jz ~ U[-1, 1], one
    field h ~ U[-0.5, 0.5] per instance, n ~ U{n_lo..n_hi}; BasicEntangling
    ansatz with L layers (P = 2 n L) and angles ~ U[-pi, pi]."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        n = rng.randint(n_lo, n_hi)
        jx = [rng.uniform(-1.0, 1.0) for _ in range(n - 1)]
        jy = [rng.uniform(-1.0, 1.0) for _ in range(n - 1)]
        jz = [rng.uniform(-1.0, 1.0) for _ in range(n - 1)]
        h = rng.uniform(-0.5, 0.5)
        theta = np.array([rng.uniform(-math.pi, math.pi) for _ in range(2 * n * layers)])
        out.append({"n": n, "jx": np.array(jx), "jy": np.array(jy), "jz": np.array(jz),
                    "h": h, "theta": theta, "layers": layers})
    return out


def disordered_chains(count: int, seed: int, n_lo=12, n_hi=16, disorder=0.2, layers=4):
    """Learned-form workload: disordered XYZ open chains.  Per chain, mean
    couplings (Jx, Jy, Jz) ~ U[-1, 1] and a field h ~ U[-0.5, 0.5]; per bond,
    J_b = J + disorder * U[-1, 1] for each axis; n ~ U{n_lo..n_hi}.  Records
    have the heisenberg_instances() layout (theta: random angles U[-pi, pi])."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        n = rng.randint(n_lo, n_hi)
        mx, my, mz = (rng.uniform(-1.0, 1.0) for _ in range(3))
        h = rng.uniform(-0.5, 0.5)
        jx = [mx + disorder * rng.uniform(-1.0, 1.0) for _ in range(n - 1)]
        jy = [my + disorder * rng.uniform(-1.0, 1.0) for _ in range(n - 1)]
        jz = [mz + disorder * rng.uniform(-1.0, 1.0) for _ in range(n - 1)]
        theta = np.array([rng.uniform(-math.pi, math.pi) for _ in range(2 * n * layers)])
        out.append({"n": n, "jx": np.array(jx), "jy": np.array(jy), "jz": np.array(jz),
                    "h": h, "theta": theta, "layers": layers})
    return out


def heisenberg_terms(n, jx, jy, jz, h) -> np.ndarray:
    """Packed Pauli terms of sum_b (Jx XX + Jy YY + Jz ZZ)_b + h sum_i Z_i."""
    terms = []
    for b in range(n - 1):
        m = (1 << (n - 1 - b)) | (1 << (n - 2 - b))
        terms.append((jx[b], m, 0, 0))
        terms.append((jy[b], m, m, 2))
        terms.append((jz[b], 0, m, 0))
    if h != 0.0:
        for i in range(n):
            terms.append((h, 0, 1 << (n - 1 - i), 0))
    arr = np.zeros(len(terms), dtype=abi.TERM_DTYPE)
    for k, (c, x, z, ny) in enumerate(terms):
        arr[k]["coefficient"] = c
        arr[k]["xmask"] = np.uint64(x)
        arr[k]["zmask"] = np.uint64(z)
        arr[k]["ny"] = ny
    return arr


def basic_entangling_template(n: int, layers: int) -> np.ndarray:
    """VariationalQuantumCircuit BasicEntangling as a parameterised gate list
    (src/qml/vqc.rs:158-170): per layer RY(p), RZ(p+1) on each qubit, then the
    CNOT(i, i+1) ladder."""
    recs = []
    p = 0
    for _ in range(layers):
        r = abi.empty_gates(2 * n)
        r["kind"][0::2] = abi.RY
        r["kind"][1::2] = abi.RZ
        r["q"][0::2, 0] = np.arange(n)
        r["q"][1::2, 0] = np.arange(n)
        r["param"][:, 0] = p + np.arange(2 * n)
        p += 2 * n
        recs.append(r)
        c = abi.empty_gates(n - 1)
        c["kind"] = abi.CNOT
        c["q"][:, 0] = np.arange(n - 1)
        c["q"][:, 1] = np.arange(1, n)
        recs.append(c)
    return np.concatenate(recs)

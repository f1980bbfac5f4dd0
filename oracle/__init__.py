"""CPU parity oracle for the LogosQ dense path -- TEST INFRASTRUCTURE ONLY.

A C++ restatement of the reference's CPU loops (oracle/logosq_oracle.cpp),
compiled with gcc into oracle/_build/liblogosq_oracle.so and called through
ctypes.  Only the test suite, the smoke check and the CPU-baseline leg of the
benchmark import this package; the product library never links or calls it.

Parity pins: tests/test_oracle_golden.py checks this oracle against the
known-answer assertions of the reference's own tests (read as text from the
reference's tests/*.rs) and against numpy; see logosq_oracle.cpp's header.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

from logosq_b200 import abi

HERE = Path(__file__).resolve().parent
SRCS = [HERE / "logosq_oracle.cpp", HERE / "mlp_oracle.cpp"]
BUILD = HERE / "_build"
LIB = BUILD / "liblogosq_oracle.so"

CXXFLAGS = ["-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared"]


def build(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    hdr = HERE.parent / "include" / "logosq_b200.h"
    newest = max([s.stat().st_mtime for s in SRCS] + [hdr.stat().st_mtime])
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        subprocess.run(["g++", *CXXFLAGS, *map(str, SRCS), "-o", str(LIB)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        lb = C.CDLL(str(LIB))
        PD, PG, PT = C.POINTER(C.c_double), C.POINTER(abi.LqGate), C.POINTER(abi.LqPauliTerm)
        PF = C.POINTER(C.c_float)
        sig = {
            "or_set_threads": (None, [C.c_int]),
            "or_get_threads": (C.c_int, []),
            "or_max_threads": (C.c_int, []),
            "or_apply_gate": (None, [PD, C.c_int, PG, PD]),
            "or_apply_circuit": (None, [PD, C.c_int, PG, C.c_int, PD]),
            "or_normalize": (None, [PD, C.c_int]),
            "or_norm_sqr": (C.c_double, [PD, C.c_int]),
            "or_probabilities": (None, [PD, C.c_int, PD]),
            "or_inner_product": (None, [PD, PD, C.c_int, PD]),
            "or_pauli_term": (C.c_double, [PD, C.c_int, PT, C.c_int]),
            "or_expectation": (C.c_double, [PD, C.c_int, PT, C.c_int, C.c_int]),
            "or_heisenberg_energy": (C.c_double, [PD, C.c_int, C.c_double, C.c_double,
                                                  C.c_double, C.c_double]),
            "or_ansatz_energy": (C.c_double, [C.c_int, PG, C.c_int, PD, PT, C.c_int, C.c_int]),
            "or_parameter_shift": (None, [C.c_int, PG, C.c_int, PD, C.c_int, PT, C.c_int, C.c_int,
                                          C.c_double, PD]),
            "or_finite_difference": (None, [C.c_int, PG, C.c_int, PD, C.c_int, PT, C.c_int,
                                            C.c_int, C.c_double, PD]),
            "or_vqe_adam": (C.c_int, [C.c_int, PG, C.c_int, PD, C.c_int, PT, C.c_int, C.c_int,
                                      C.c_double, C.c_int, C.c_double, PD, PD]),
            "or_apply_dense": (None, [PD, C.c_int, PD]),
            "or_mlp_num_params": (C.c_int64, [C.c_int] * 4),
            "or_mlp_forward": (None, [C.c_int] * 4 + [PF, PF, C.c_int, PD]),
            "or_mlp_loss_grad": (C.c_double, [C.c_int] * 4 + [PD, PF, PF, PF, C.c_int, PD]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lb, name)
            f.restype = res
            f.argtypes = args
        _lib = lb
    return _lib


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_threads(t: int) -> None:
    """1 = faithful mode (serial where the reference is serial); >1 threaded."""
    lib().or_set_threads(int(t))


def max_threads() -> int:
    return lib().or_max_threads()


def zero_state(n: int) -> np.ndarray:
    v = np.zeros(1 << n, dtype=np.complex128)
    v[0] = 1.0
    return v


def apply_circuit(psi: np.ndarray, gates: np.ndarray, theta=None) -> np.ndarray:
    """In place on psi (complex128, contiguous); returns psi."""
    assert psi.dtype == np.complex128 and psi.flags["C_CONTIGUOUS"]
    n = int(np.log2(len(psi)))
    th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
    lib().or_apply_circuit(_pd(psi.view(np.float64)), n, abi.gate_ptr(gates), len(gates),
                           None if th is None else _pd(th))
    return psi


def normalize(psi):
    lib().or_normalize(_pd(psi.view(np.float64)), int(np.log2(len(psi))))
    return psi


def norm_sqr(psi) -> float:
    return lib().or_norm_sqr(_pd(psi.view(np.float64)), int(np.log2(len(psi))))


def probabilities(psi):
    out = np.empty(len(psi), dtype=np.float64)
    lib().or_probabilities(_pd(psi.view(np.float64)), int(np.log2(len(psi))), _pd(out))
    return out


def inner_product(a, b) -> complex:
    out = np.zeros(2)
    lib().or_inner_product(_pd(a.view(np.float64)), _pd(b.view(np.float64)),
                           int(np.log2(len(a))), _pd(out))
    return complex(out[0], out[1])


def expectation(psi, terms: np.ndarray, y_convention: int = abi.Y_REFERENCE) -> float:
    return lib().or_expectation(_pd(psi.view(np.float64)), int(np.log2(len(psi))),
                                abi.term_ptr(terms), len(terms), y_convention)


def heisenberg_energy(psi, jx, jy, jz, h) -> float:
    return lib().or_heisenberg_energy(_pd(psi.view(np.float64)), int(np.log2(len(psi))),
                                      jx, jy, jz, h)


def ansatz_energy(n, gates, theta, terms, y_convention=abi.Y_REFERENCE) -> float:
    th = np.ascontiguousarray(theta, dtype=np.float64)
    return lib().or_ansatz_energy(n, abi.gate_ptr(gates), len(gates), _pd(th), abi.term_ptr(terms),
                                  len(terms), y_convention)


def parameter_shift(n, gates, theta, terms, shift=np.pi / 2, y_convention=abi.Y_REFERENCE):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    g = np.zeros(len(th))
    lib().or_parameter_shift(n, abi.gate_ptr(gates), len(gates), _pd(th), len(th),
                             abi.term_ptr(terms), len(terms), y_convention, shift, _pd(g))
    return g


def finite_difference(n, gates, theta, terms, eps=1e-7, y_convention=abi.Y_REFERENCE):
    th = np.ascontiguousarray(theta, dtype=np.float64)
    g = np.zeros(len(th))
    lib().or_finite_difference(n, abi.gate_ptr(gates), len(gates), _pd(th), len(th),
                               abi.term_ptr(terms), len(terms), y_convention, eps, _pd(g))
    return g


def vqe_adam(n, gates, theta0, terms, lr=0.1, max_iter=100, tol=1e-6,
             y_convention=abi.Y_REFERENCE):
    th = np.array(theta0, dtype=np.float64)
    hist = np.zeros(max_iter + 1)
    fv = C.c_double()
    k = lib().or_vqe_adam(n, abi.gate_ptr(gates), len(gates), _pd(th), len(th),
                          abi.term_ptr(terms), len(terms), y_convention, lr, max_iter, tol,
                          _pd(hist), C.byref(fv))
    return th, fv.value, hist[:k]


def apply_dense(psi, matrix):
    m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
    lib().or_apply_dense(_pd(psi.view(np.float64)), int(np.log2(len(psi))),
                         _pd(m.view(np.float64)))
    return psi


def _pf(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def mlp_num_params(in_dim, hidden, depth, out_dim) -> int:
    return int(lib().or_mlp_num_params(in_dim, hidden, depth, out_dim))


def mlp_forward(shape, params, x):
    """FP64 forward pass of the warm-start network (mlp_oracle.cpp) for float32
    parameters and inputs."""
    in_dim, hidden, depth, out_dim = shape
    p = np.ascontiguousarray(params, dtype=np.float32)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    y = np.zeros((len(xx), out_dim))
    lib().or_mlp_forward(in_dim, hidden, depth, out_dim, _pf(p), _pf(xx), len(xx), _pd(y))
    return y


def mlp_loss_grad(shape, params, x, target, mask):
    """FP64 periodic angle loss and its gradient w.r.t. the flat parameters."""
    in_dim, hidden, depth, out_dim = shape
    p = np.ascontiguousarray(params, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(target, dtype=np.float32)
    m = np.ascontiguousarray(mask, dtype=np.float32)
    g = np.zeros(len(p))
    loss = lib().or_mlp_loss_grad(in_dim, hidden, depth, out_dim, _pd(p), _pf(xx), _pf(t),
                                  _pf(m), len(xx), _pd(g))
    return loss, g


def dense_hamiltonian(n: int, terms: np.ndarray) -> np.ndarray:
    """Real dense matrix of a Pauli sum whose terms all carry an even number of
    Y factors (textbook Pauli matrices; for such terms the reference's Y sign
    convention gives the same operator).  Qubit q is bit n-1-q."""
    N = 1 << n
    idx = np.arange(N, dtype=np.int64)
    H = np.zeros((N, N))
    for t in terms:
        x, z, ny = int(t["xmask"]), int(t["zmask"]), int(t["ny"])
        assert ny % 2 == 0, "real Hamiltonian needs an even number of Y per term"
        parity = np.zeros(N, dtype=np.int64)
        zz = idx & z
        while zz.any():
            parity ^= zz & 1
            zz >>= 1
        phase = -1.0 if ny % 4 == 2 else 1.0
        H[idx ^ x, idx] += float(t["coefficient"]) * phase * (1.0 - 2.0 * parity)
    return H


# ---------------------------------------------------------------------------
# Noise models: numpy restatement of src/noise/mod.rs (bit `qubit` = 1 << qubit)
# ---------------------------------------------------------------------------
def noise_pauli(psi, qubit: int, pauli: int):
    """apply_x_error / apply_y_error / apply_z_error (src/noise/mod.rs:337-380)."""
    idx = np.arange(len(psi))
    j = idx ^ (1 << qubit)
    bit = (idx >> qubit) & 1
    if pauli == 1:
        return psi[j].copy()
    if pauli == 2:  # new[i] = -i psi[j] if bit(i) else +i psi[j]
        return np.where(bit == 1, -1j, 1j) * psi[j]
    return np.where(bit == 1, -psi, psi)


def noise_amplitude_damping(psi, gamma: float, qubits):
    """AmplitudeDampingNoise::apply (src/noise/mod.rs:108-146): one zero vector,
    every target qubit's K0 + K1 terms added into it, then normalised."""
    new = np.zeros_like(psi)
    idx = np.arange(len(psi))
    for q in qubits:
        bit = (idx >> q) & 1
        zero = bit == 0
        new[zero] += psi[zero]
        one = ~zero
        new[one] += psi[one] * math.sqrt(1.0 - gamma)
        np.add.at(new, idx[one] & ~(1 << q), psi[one] * math.sqrt(gamma))
    return new / np.sqrt(np.sum(np.abs(new) ** 2))


def noise_phase_damping(psi, lam: float, qubits):
    """PhaseDampingNoise::apply (src/noise/mod.rs:173-210): each target qubit
    rewrites the vector from the input, so the last one's damping survives;
    then normalised."""
    idx = np.arange(len(psi))
    new = psi.copy()
    for q in qubits:
        new = psi.copy()
        new[((idx >> q) & 1) == 1] *= math.sqrt(1.0 - lam)
    return new / np.sqrt(np.sum(np.abs(new) ** 2))


# ---------------------------------------------------------------------------
# Shot sampling.  The reference's measure (src/states/mod.rs:180-185) and
# measure_shots_parallel (:244-258) draw each shot with rand 0.8's WeightedIndex:
# the running sums of |psi_i|^2, a uniform u in [0, total), and the first index
# whose running sum exceeds u.  The engine keeps that rule with its own
# counter-based uniforms (SplitMix64 of the shot number) and running sums in a
# fixed parallel order; this restatement reproduces both bit for bit, so the
# sampled indices can be compared exactly.
# ---------------------------------------------------------------------------
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return x ^ (x >> np.uint64(31))


def _scan_chunks(v: np.ndarray):
    """One level of the engine's fixed-order inclusive scan: chunks of 1024
    values, 256 threads x 4 running sums, a Kogge-Stone scan of the thread
    totals inside each 32-lane warp, an in-order exclusive scan of the 8 warp
    totals, cdf = (W_warp + incl_{t-1}) + s_j."""
    N = len(v)
    nc = -(-N // 1024)
    x = np.zeros(nc * 1024)
    x[:N] = v
    x = x.reshape(nc, 8, 32, 4)
    s = np.cumsum(x, axis=3)                       # sequential, left to right
    incl = s[..., 3].copy()                        # (nc, 8, 32)
    for off in (1, 2, 4, 8, 16):
        old = incl.copy()
        incl[..., off:] = old[..., :-off] + old[..., off:]
    excl = np.zeros_like(incl)
    excl[..., 1:] = incl[..., :-1]
    wt = incl[..., 31]                             # (nc, 8) warp totals
    W = np.zeros_like(wt)
    run = np.zeros(nc)
    for w in range(8):
        W[:, w] = run
        run = run + wt[:, w]
    off = W[..., None] + excl                      # (nc, 8, 32)
    cdf = off[..., None] + s
    cdf = cdf.reshape(-1)
    return cdf[:N], cdf.reshape(nc, 1024)[:, -1].copy()


def sampling_cdf(psi: np.ndarray) -> np.ndarray:
    """The engine's cumulative probabilities of psi, value for value."""
    p = psi.real * psi.real + psi.imag * psi.imag   # two products, one sum: no FMA
    return _scan(p)


def _scan(v: np.ndarray) -> np.ndarray:
    """Chunk scans, chunk totals scanned the same way, base + value."""
    cdf, tot = _scan_chunks(v)
    if len(tot) > 1:
        incl = _scan(tot)
        c = np.arange(len(cdf)) // 1024
        later = c >= 1
        cdf[later] = incl[c[later] - 1] + cdf[later]
    return cdf


def sample_indices(psi: np.ndarray, n_shots: int, seed: int) -> np.ndarray:
    """Shot s draws u = (r >> 11) * 2^-53 * total with r = SplitMix64(seed xor
    SplitMix64(s)) and returns the first index whose running sum exceeds u."""
    cdf = sampling_cdf(np.ascontiguousarray(psi, dtype=np.complex128))
    total = cdf[-1]
    s = np.arange(n_shots, dtype=np.uint64)
    r = _splitmix64(np.uint64(seed) ^ _splitmix64(s))
    u = (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) * total
    idx = np.searchsorted(cdf, u, side="right")
    return np.minimum(idx, len(cdf) - 1).astype(np.uint64)

"""Learned warm start for VQE on XYZ chains.

A fully connected network (couplings -> BasicEntangling angles) trained in
FP32 on the device by the engine's own kernels (lq_mlp_*), first on VQE optima
that the batched parameter-shift engine (lq_batch_*) generates, then on the
simulator's energy itself; exact ground energies come from the engine's FP64
Lanczos (lq_lanczos_ground_energy).

No reference counterpart: the reference's VQE (src/optimization/vqe.rs:69-88)
starts from caller-supplied angles and its optimizers
(src/optimization/optimizer.rs) iterate from there.  This module produces the
starting angles; plain random-init VQE stays the fallback.

Layout of one sample:
  features  float32[46]: (Jx_b, Jy_b, Jz_b) for bonds b = 0..14 (zero padded
            beyond the chain's n-1 bonds), then the field h;
  angles    float32[128]: the 8n BasicEntangling L=4 angles (zero padded);
  mask      float32[128]: 1 on the first 8n entries.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import abi, workloads
from ._lib import call, lib

MAX_BONDS = 15
IN_DIM = 3 * MAX_BONDS + 1
OUT_DIM = 128
HIDDEN = 256
DEPTH = 3
LAYERS = 4


def features(rec) -> np.ndarray:
    f = np.zeros(IN_DIM, dtype=np.float32)
    nb = rec["n"] - 1
    if nb > MAX_BONDS:
        raise ValueError(f"chain of {rec['n']} qubits exceeds {MAX_BONDS} bonds")
    f[0:3 * nb:3] = rec["jx"]
    f[1:3 * nb:3] = rec["jy"]
    f[2:3 * nb:3] = rec["jz"]
    f[IN_DIM - 1] = rec["h"]
    return f


def angle_mask(n: int) -> np.ndarray:
    m = np.zeros(OUT_DIM, dtype=np.float32)
    m[:2 * LAYERS * n] = 1.0
    return m


def fixed_start(n: int, seed: int = 7, scale: float = 0.1) -> np.ndarray:
    """The deterministic small-angle start used to generate training optima:
    the same U[-scale, scale] vector (SplitMix64 stream) for every chain of n
    qubits, so that an optimum depends as smoothly as possible on the couplings."""
    return workloads.uniform_stream(seed * 1000 + n, 2 * LAYERS * n, -scale, scale)


def random_start(n: int, rng: np.random.Generator) -> np.ndarray:
    return rng.uniform(-math.pi, math.pi, 2 * LAYERS * n)


def chain_terms(rec) -> np.ndarray:
    return workloads.heisenberg_terms(rec["n"], rec["jx"], rec["jy"], rec["jz"], rec["h"])


class WarmStartMLP:
    """in_dim -> hidden (x depth, GELU) -> out_dim on the device (FP32)."""

    def __init__(self, in_dim=IN_DIM, hidden=HIDDEN, depth=DEPTH, out_dim=OUT_DIM, seed=1):
        self.shape = (in_dim, hidden, depth, out_dim)
        self.val_hist = []
        h = C.c_void_p()
        call("lq_mlp_create", in_dim, hidden, depth, out_dim, seed, C.byref(h))
        self._h = h
        n = C.c_int64()
        call("lq_mlp_num_params", h, C.byref(n))
        self.num_params = n.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().lq_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _pf(a):
        return a.ctypes.data_as(C.POINTER(C.c_float))

    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params, dtype=np.float32)
        call("lq_mlp_get_params", self._h, self._pf(p), self.num_params)
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        call("lq_mlp_set_params", self._h, self._pf(p), len(p))

    def grads(self) -> np.ndarray:
        g = np.zeros(self.num_params, dtype=np.float32)
        call("lq_mlp_get_grads", self._h, self._pf(g), self.num_params)
        return g

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((len(x), self.shape[3]), dtype=np.float32)
        call("lq_mlp_forward", self._h, self._pf(x), len(x), self._pf(y))
        return y

    def loss_grad(self, x, target, mask) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(target, dtype=np.float32)
        m = np.ascontiguousarray(mask, dtype=np.float32)
        loss = C.c_double()
        call("lq_mlp_loss_grad", self._h, self._pf(x), self._pf(t), self._pf(m), len(x),
             C.byref(loss))
        return loss.value

    def backward(self, x, dy) -> None:
        """Parameter gradient for a given dL/dy at inputs x (kept on the device)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        d = np.ascontiguousarray(dy, dtype=np.float32)
        call("lq_mlp_backward", self._h, self._pf(x), self._pf(d), len(x))

    def adam_step(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8) -> None:
        call("lq_mlp_adam_step", self._h, lr, beta1, beta2, eps)

    def angle_loss(self, X, T, M) -> float:
        """Periodic angle loss of the current parameters (no update)."""
        Y = self.forward(X).astype(np.float64)
        return float(np.sum(M * (1.0 - np.cos(Y - T))) / np.sum(M))

    def fit(self, X, T, M, epochs=200, batch=256, lr=1e-3, seed=0, val_frac=0.0, log=None):
        """First training stage: minibatch Adam on the periodic angle loss
        against VQE optima; returns the per-epoch mean training loss.  With
        val_frac > 0 that share of the samples is held out and the parameters of
        the epoch with the lowest held-out loss are kept (early stopping);
        self.val_hist then holds the held-out losses."""
        call("lq_mlp_reset_adam", self._h)
        rng = np.random.default_rng(seed)
        nval = int(len(X) * val_frac)
        perm = rng.permutation(len(X))
        vi, ti = perm[:nval], perm[nval:]
        hist, self.val_hist = [], []
        best, best_p = math.inf, None
        for ep in range(epochs):
            order = ti[rng.permutation(len(ti))]
            tot, cnt = 0.0, 0
            for s in range(0, len(order), batch):
                idx = order[s:s + batch]
                tot += self.loss_grad(X[idx], T[idx], M[idx]) * len(idx)
                cnt += len(idx)
                self.adam_step(lr)
            hist.append(tot / cnt)
            if nval:
                v = self.angle_loss(X[vi], T[vi], M[vi])
                self.val_hist.append(v)
                if v < best:
                    best, best_p = v, self.params()
            if log and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
                log(f"epoch {ep}: loss {hist[-1]:.5f}" +
                    (f" held-out {self.val_hist[-1]:.5f}" if nval else ""))
        if best_p is not None:
            self.set_params(best_p)
        return hist

    def energy_train(self, recs, steps, lr=3e-4, chunk=256, log=None):
        """Second training stage: the loss is the mean VQE energy of the
        network's angles, E(net(x)), judged by the simulator itself.  Each step
        takes one chunk of chains, evaluates E and dE/dtheta for all of them in
        one batched parameter-shift launch (lq_batch_gradients) and
        back-propagates dE/dtheta through the network.  Returns the mean energy
        per step."""
        from .batch import heisenberg_batch
        call("lq_mlp_reset_adam", self._h)
        chunks = [recs[i:i + chunk] for i in range(0, len(recs), chunk)]
        engines = [heisenberg_batch(c, layers=LAYERS) for c in chunks]
        feats = [np.stack([features(r) for r in c]) for c in chunks]
        hist = []
        try:
            for s in range(steps):
                k = s % len(chunks)
                c, b, X = chunks[k], engines[k], feats[k]
                Y = self.forward(X)
                th = np.concatenate([Y[i, :2 * LAYERS * r["n"]] for i, r in enumerate(c)])
                E, g = b.gradients(th.astype(np.float64))
                dY = np.zeros_like(Y)
                for i, gi in enumerate(b.split(g)):
                    dY[i, :len(gi)] = gi / len(c)
                self.backward(X, dY)
                self.adam_step(lr)
                hist.append(float(E.mean()))
                if log and (s % max(1, steps // 10) == 0 or s == steps - 1):
                    log(f"energy step {s}: mean E {hist[-1]:.5f}")
        finally:
            for b in engines:
                b.close()
        return hist

    def warm_start(self, recs) -> list[np.ndarray]:
        y = self.forward(np.stack([features(r) for r in recs]))
        return [y[i, :2 * LAYERS * r["n"]].astype(np.float64) for i, r in enumerate(recs)]


def lanczos_ground_energy(n: int, terms: np.ndarray, max_iter=300, tol=1e-12, seed=11):
    """(E0, iterations) from the device's FP64 Lanczos."""
    e0, it = C.c_double(), C.c_int()
    t = np.ascontiguousarray(terms)
    call("lq_lanczos_ground_energy", n, abi.term_ptr(t), len(t), max_iter, tol, seed,
         C.byref(e0), C.byref(it))
    return e0.value, it.value


def batched_vqe(recs, starts, iters, lr=0.05, chunk=256):
    """Adam VQE for every chain at once with the batched parameter-shift engine,
    `chunk` chains per launch.  One iteration = one batched energy+gradient
    call followed by an Adam update (the update rule of Adam::minimize,
    src/optimization/optimizer.rs:139-223, without its early exit so every
    chain runs `iters` steps).  Returns (final angles, energy trace
    [len(recs) x (iters+1)] where column k is the energy after k updates,
    seconds per iteration of each chunk)."""
    from .batch import heisenberg_batch
    out = [None] * len(recs)
    E = np.zeros((len(recs), iters + 1))
    sec = []
    for c0 in range(0, len(recs), chunk):
        sub = recs[c0:c0 + chunk]
        b = heisenberg_batch(sub, layers=LAYERS)
        th = np.concatenate([np.asarray(s, dtype=np.float64) for s in starts[c0:c0 + chunk]])
        m = np.zeros_like(th)
        v = np.zeros_like(th)
        b.gradients(th)  # tuning + graph capture outside the timing
        t0 = time.perf_counter()
        for it in range(1, iters + 1):
            e, g = b.gradients(th)
            E[c0:c0 + len(sub), it - 1] = e
            m = 0.9 * m + 0.1 * g
            v = 0.999 * v + 0.001 * g * g
            th -= lr * (m / (1 - 0.9 ** it)) / (np.sqrt(v / (1 - 0.999 ** it)) + 1e-8)
        e, _ = b.gradients(th)
        sec.append((time.perf_counter() - t0) / (iters + 1))
        E[c0:c0 + len(sub), iters] = e
        for i, part in enumerate(b.split(th)):
            out[c0 + i] = part.copy()
        b.close()
    return out, E, sec


def optimum_dataset(recs, iters=300, lr=0.05, chunk=256):
    """(X, T, M, final energies, seconds per iteration) from batched VQE runs
    started at fixed_start(n)."""
    starts = [fixed_start(r["n"]) for r in recs]
    th, E, sec = batched_vqe(recs, starts, iters, lr, chunk)
    X = np.stack([features(r) for r in recs])
    T = np.zeros((len(recs), OUT_DIM), dtype=np.float32)
    M = np.stack([angle_mask(r["n"]) for r in recs])
    for i, t in enumerate(th):
        # wrap to (-pi, pi]: the energy is 2*pi periodic in every angle
        T[i, :len(t)] = np.angle(np.exp(1j * t))
    return X, T, M, E[:, -1], sec


def iterations_to(trace: np.ndarray, target: np.ndarray, tol: float) -> np.ndarray:
    """First iteration index whose energy is within tol of target (per row);
    trace.shape[1] where never reached."""
    hit = trace - target[:, None] < tol
    return np.where(hit.any(axis=1), hit.argmax(axis=1), trace.shape[1])

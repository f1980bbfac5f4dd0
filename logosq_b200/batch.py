"""Batched parameter-shift gradients: many VQE instances of uneven qubit counts,
all 2P+1 circuits of every instance in one persistent, CUDA-graph-captured
launch (lq_batch_*).  Mirrors running ParameterShift::compute_gradient
(src/optimization/gradient.rs:44-78) plus the VQE objective
(src/optimization/vqe.rs:63-67) for each instance."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi
from ._lib import call, lib


class BatchedParameterShift:
    """instances: list of (num_qubits, template_gates, nparams, terms) where the
    template is a parameterised gate array (abi.GATE_DTYPE) and terms a packed
    Pauli-term array (abi.TERM_DTYPE)."""

    def __init__(self, instances):
        self._keep = []
        arr = (abi.LqVqeInstance * len(instances))()
        self.nparams = []
        for i, (n, gates, nparams, terms) in enumerate(instances):
            g = np.ascontiguousarray(gates)
            t = np.ascontiguousarray(terms)
            self._keep += [g, t]
            arr[i].num_qubits = int(n)
            arr[i].nops = len(g)
            arr[i].ops = abi.gate_ptr(g)
            arr[i].nparams = int(nparams)
            arr[i].nterms = len(t)
            arr[i].terms = abi.term_ptr(t)
            self.nparams.append(int(nparams))
        self._arr = arr
        h = C.c_void_p()
        call("lq_batch_create", arr, len(instances), C.byref(h))
        self._h = h
        self.ninst = len(instances)
        self.offsets = np.concatenate([[0], np.cumsum(self.nparams)]).astype(int)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().lq_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def gradients(self, theta_all, shift: float = math.pi / 2):
        """theta_all: concatenated parameter vectors.  Returns (energies[ninst],
        gradient[total params])."""
        th = np.ascontiguousarray(theta_all, dtype=np.float64)
        assert len(th) == self.offsets[-1]
        e = np.zeros(self.ninst)
        g = np.zeros(len(th))
        call("lq_batch_gradients", self._h, abi.f64_ptr(th), float(shift), abi.f64_ptr(e),
             abi.f64_ptr(g))
        return e, g

    def split(self, flat):
        return [flat[self.offsets[i]:self.offsets[i + 1]] for i in range(self.ninst)]

    def tuning(self):
        a, b = C.c_int(), C.c_int()
        call("lq_batch_tuning", self._h, C.byref(a), C.byref(b))
        c, d = C.c_int(), C.c_uint64()
        call("lq_batch_prefix_info", self._h, C.byref(c), C.byref(d))
        return {"smem_max_qubits": a.value, "tile_bits": b.value,
                "shared_prefixes": bool(c.value), "checkpoint_bytes": d.value}


def heisenberg_batch(instances, layers=4):
    """BatchedParameterShift over workloads.heisenberg_instances() records with
    the BasicEntangling ansatz."""
    from . import workloads as W
    specs = []
    for r in instances:
        n = r["n"]
        specs.append((n, W.basic_entangling_template(n, layers), 2 * n * layers,
                      W.heisenberg_terms(n, r["jx"], r["jy"], r["jz"], r["h"])))
    return BatchedParameterShift(specs)

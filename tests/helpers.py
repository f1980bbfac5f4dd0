"""Shared helpers: build circuits from the golden JSON op lists, run them on the
engine or on the oracle, and evaluate the reference's assertions."""
from __future__ import annotations

import cmath
import json
import math
from pathlib import Path

import numpy as np

from logosq_b200 import Circuit, abi, qft
from logosq_b200.optimization import Pauli, PauliTerm, pack_terms

GOLDEN = Path(__file__).resolve().parent / "golden"


def known_answers():
    return json.loads((GOLDEN / "known_answers.json").read_text())


def perm_matrix(entries, dim):
    """dim x dim matrix from [row, col] entries equal to 1, or [row, col, value]
    entries with a real value."""
    m = np.zeros((dim, dim), dtype=np.complex128)
    for e in entries:
        m[e[0], e[1]] = e[2] if len(e) > 2 else 1.0
    return m


def build(n, ops) -> Circuit:
    """Circuit from builder calls, with the reference's builder semantics
    (Circuit::x/h are dense builders; cnot/rx/... are gate structs)."""
    c = Circuit(n)
    for op in ops:
        name, args = op[0], op[1:]
        if name == "qft":
            c.compose(qft.create_circuit(n))
        elif name == "iqft":
            c.compose(qft.create_inverse_circuit(n))
        elif name == "dense":
            c.add_matrix_gate(perm_matrix(args[0], 1 << n), list(range(n)), "dense")
        else:
            getattr(c, name)(*args)
    return c


def oracle_run(circuit: Circuit, psi=None) -> np.ndarray:
    import oracle
    n = circuit.num_qubits()
    v = oracle.zero_state(n) if psi is None else np.array(psi, dtype=np.complex128)
    for kind, seg in circuit.segments():
        if kind == "dense":
            oracle.apply_dense(v, seg)
        else:
            oracle.apply_circuit(v, seg)
    return v


def gpu_run(circuit: Circuit, psi=None, mode=abi.EXEC_FUSED) -> np.ndarray:
    from logosq_b200 import State
    n = circuit.num_qubits()
    st = State.zero_state(n)
    if psi is not None:
        st.set_vector(psi)
    circuit.execute(st, mode=mode)
    v = st.vector()
    st.close()
    return v


def check_case(v: np.ndarray, checks, run) -> list[str]:
    """Evaluate the reference assertions on amplitudes v; returns failures."""
    bad = []
    probs = np.abs(v) ** 2
    for c in checks:
        kind = c[0]
        ok = True
        if kind == "prob_gt":
            ok = probs[c[1]] > c[2]
        elif kind == "prob_lt":
            ok = probs[c[1]] < c[2]
        elif kind == "prob_eq":
            ok = abs(probs[c[1]] - c[2]) < c[3]
        elif kind == "abs_lt":
            ok = abs(v[c[1]]) < c[2]
        elif kind == "abs_eq":
            ok = abs(abs(v[c[1]]) - c[2]) < c[3]
        elif kind == "arg_eq":
            ok = abs(cmath.phase(v[c[1]]) - c[2]) < c[3]
        elif kind == "amp_eq":
            ok = abs(v[c[1]] - complex(*c[2])) < c[3]
        elif kind == "imag_lt":
            ok = abs(v[c[1]].imag) < c[2]
        elif kind == "real_gt":
            ok = v[c[1]].real > c[2]
        elif kind == "norm_eq":
            ok = abs(probs.sum() - c[1]) < c[2]
        elif kind == "nonzero_count_gt":
            ok = int((probs > c[1]).sum()) > c[2]
        elif kind == "absarg_ratio_eq":
            ok = abs(abs(cmath.phase(v[c[1]] / v[c[2]])) - c[3]) < c[4]
        elif kind == "phase_mod_eq":
            d = abs(c[2] - cmath.phase(v[c[1]])) % (2 * math.pi)
            ok = min(d, 2 * math.pi - d) < c[3]
        elif kind == "same_as":
            w = run(c[1])
            ok = np.abs(v - w).max() < c[2]
        elif kind == "expect_matrix":
            m = np.array([complex(*e) for e in c[1]]).reshape(2, 2)
            ok = abs(np.vdot(v, m @ v).real - c[2]) < c[3]
        else:
            raise ValueError(kind)
        if not ok:
            bad.append(str(c))
    return bad


def terms_from_strings(n, spec) -> np.ndarray:
    terms = []
    for coef, s in spec:
        terms.append(PauliTerm(coef, [getattr(Pauli, ch) for ch in s]))
    return pack_terms(terms, n)


def random_state(n, seed):
    from logosq_b200.workloads import gaussian_state
    return gaussian_state(n, seed)


def numpy_apply(v, n, matrix, qubits):
    """Reference-independent check: apply a k-qubit matrix by tensor reshaping
    (qubit q is axis q of the (2,)*n view: big-endian)."""
    k = len(qubits)
    t = v.reshape((2,) * n)
    m = np.asarray(matrix).reshape((2,) * (2 * k))
    out = np.tensordot(m, t, axes=(list(range(k, 2 * k)), list(qubits)))
    # tensordot puts the k new axes first; move them back into place
    out = np.moveaxis(out, list(range(k)), list(qubits))
    return out.reshape(-1)

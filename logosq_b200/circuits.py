"""`Circuit`: the drop-in for src/circuits/*.rs.

A circuit is an ordered list of packed gate descriptors.  `execute(state)`
submits the whole list in one call (lq_apply_circuit), where the engine plans
it into fused shared-memory passes; `execute(state, mode=EXEC_PER_GATE)` runs one
sweep per gate in order (the reference's loop, src/circuits/mod.rs:362-373).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import LogosQError, call
from .gates import Gate, MatrixGate, make_desc
from . import gates as G


class Operation:
    """One operation (src/circuits/mod.rs:29-33): a descriptor, or a full dense
    matrix (MatrixGate) which runs as its own dense kernel."""

    __slots__ = ("desc", "dense", "_qubits", "_name")

    def __init__(self, desc, qubits, name, dense=None):
        self.desc = desc
        self.dense = dense
        self._qubits = list(qubits)
        self._name = name

    def qubits(self):
        """Operation::qubits (src/circuits/mod.rs:51-53)."""
        return self._qubits

    def name(self):
        """Operation::name (src/circuits/mod.rs:56-58)."""
        return self._name

    def __repr__(self):
        # Debug for Operation (src/circuits/mod.rs:61-65)
        return f"{self._name}(qubits: {self._qubits})"


def _expand_single(matrix, target, n):
    """kron(I.., M, ..I) with qubit 0 leftmost (src/circuits/single_qubit.rs:12-60)."""
    eye = np.eye(2, dtype=np.complex128)
    full = matrix if target == 0 else eye
    for i in range(1, n):
        full = np.kron(full, matrix if i == target else eye)
    return full


class Circuit:
    """Mirror of `Circuit` (src/circuits/mod.rs:81-86)."""

    def __init__(self, num_qubits: int):
        self._n = int(num_qubits)
        self._ops: list[Operation] = []
        self._name: str | None = None
        self._packed: np.ndarray | None = None
        self._noise: list = []

    # -- metadata ---------------------------------------------------------
    def with_name(self, name: str) -> "Circuit":
        self._name = name
        return self

    def num_qubits(self) -> int:
        return self._n

    def num_operations(self) -> int:
        return len(self._ops)

    def operations(self):
        return list(self._ops)

    def name(self):
        return self._name

    # -- construction -----------------------------------------------------
    def _check(self, *qubits):
        for q in qubits:
            if q < 0 or q >= self._n:
                raise LogosQError(abi.LQ_ERR_QUBIT_INDEX,
                                  f"Invalid qubit index: {q} (must be < {self._n})")

    def _push(self, desc, qubits, name, dense=None):
        self._ops.append(Operation(desc, qubits, name, dense))
        self._packed = None
        return self

    def add_operation(self, gate: Gate, qubits, name: str):
        """add_operation (src/circuits/mod.rs:137-158)."""
        self._check(*qubits)
        if isinstance(gate, MatrixGate):
            return self._push(None, qubits, name, dense=gate.matrix)
        return self._push(gate.descriptor(), qubits, name)

    def add_matrix_gate(self, matrix, qubits, name: str):
        """add_matrix_gate (src/circuits/mod.rs:183-191): a full-state matrix."""
        return self.add_operation(MatrixGate(matrix), qubits, name)

    def add_single_qubit_gate(self, gate_matrix, target_qubit: int, name: str):
        """Circuit::add_single_qubit_gate (src/circuits/single_qubit.rs:12-60).

        The reference expands the 2x2 to a dense 2^n x 2^n MatrixGate, which
        then renormalises the state.  Here the 2x2 is applied by a single-qubit
        sweep followed by the same renormalisation.
        """
        m = np.asarray(gate_matrix, dtype=np.complex128)
        if m.shape != (2, 2):
            raise LogosQError(abi.LQ_ERR_GATE_MATRIX, "Gate must be a 2x2 matrix")
        self._check(target_qubit)
        return self._push(make_desc(abi.MATRIX1, [target_qubit], flags=abi.FLAG_RENORM,
                                    matrix=m), list(range(self._n)), name)

    def add_two_qubit_gate(self, gate_matrix, control: int, target: int, name: str):
        """Circuit::add_two_qubit_gate (src/circuits/two_qubits.rs:11-82)."""
        m = np.asarray(gate_matrix, dtype=np.complex128)
        if m.shape != (4, 4):
            raise LogosQError(abi.LQ_ERR_GATE_MATRIX, "Gate must be a 4x4 matrix")
        self._check(control, target)
        return self._push(make_desc(abi.MATRIX2, [control, target], flags=abi.FLAG_RENORM,
                                    matrix=m), list(range(self._n)), name)

    # dense builders (src/circuits/single_qubit.rs:63-126)
    def x(self, q): return self.add_single_qubit_gate(G.x_matrix(), q, "X")
    def y(self, q): return self.add_single_qubit_gate(G.y_matrix(), q, "Y")
    def z(self, q): return self.add_single_qubit_gate(G.z_matrix(), q, "Z")
    def h(self, q): return self.add_single_qubit_gate(G.h_matrix(), q, "H")
    def s(self, q): return self.add_single_qubit_gate(G.s_matrix(), q, "S")
    def t(self, q): return self.add_single_qubit_gate(G.t_matrix(), q, "T")
    def rx_matrix(self, q, th): return self.add_single_qubit_gate(G.rx_matrix(th), q, f"RX({th})")
    def ry_matrix(self, q, th): return self.add_single_qubit_gate(G.ry_matrix(th), q, f"RY({th})")
    def rz_matrix(self, q, th): return self.add_single_qubit_gate(G.rz_matrix(th), q, f"RZ({th})")

    # optimized struct builders (src/circuits/two_qubits.rs:85-137, three_qubits.rs)
    def cnot(self, control, target):
        self._check(control, target)
        if control == target:
            raise LogosQError(abi.LQ_ERR_INVALID_ARG, "Control and target must be different")
        return self._push(make_desc(abi.CNOT, [control, target]), [control, target], "CNOT")

    def swap(self, q1, q2):
        self._check(q1, q2)
        if q1 == q2:
            raise LogosQError(abi.LQ_ERR_INVALID_ARG, "Qubits must be different")
        return self._push(make_desc(abi.SWAP, [q1, q2]), [q1, q2], "SWAP")

    def cz(self, control, target):
        self._check(control, target)
        if control == target:
            raise LogosQError(abi.LQ_ERR_INVALID_ARG, "Control and target must be different")
        return self._push(make_desc(abi.CZ, [control, target]), [control, target], "CZ")

    def toffoli(self, c1, c2, target):
        self._check(c1, c2, target)
        if len({c1, c2, target}) != 3:
            raise LogosQError(abi.LQ_ERR_INVALID_ARG, "Control and target qubits must be different")
        return self._push(make_desc(abi.TOFFOLI, [c1, c2, target]), [c1, c2, target], "Toffoli")

    def cphase(self, control, target, angle):
        """qft::controlled_phase (src/algorithms/qft.rs:96-105): a CPhaseGate struct."""
        self._check(control, target)
        return self._push(make_desc(abi.CPHASE, [control, target], [angle]), [control, target],
                          f"CP({angle:.4f})")

    # parameterized builders (src/circuits/parameterized.rs:28-392)
    def _p1(self, kind, q, angles, name, params=None, scales=None):
        self._check(q)
        return self._push(make_desc(kind, [q], angles, params=params, scales=scales), [q], name)

    def _p2(self, kind, a, b, th, name, flags=0, params=None, scales=None):
        self._check(a, b)
        return self._push(make_desc(kind, [a, b], [th], flags=flags, params=params,
                                    scales=scales), [a, b], name)

    def rx(self, q, theta): return self._p1(abi.RX, q, [theta], "RX")
    def ry(self, q, theta): return self._p1(abi.RY, q, [theta], "RY")
    def rz(self, q, theta): return self._p1(abi.RZ, q, [theta], "RZ")
    def phase(self, q, theta): return self._p1(abi.PHASE, q, [theta], "P")
    def u3(self, q, theta, phi, lambda_): return self._p1(abi.U3, q, [theta, phi, lambda_], "U3")
    def crx(self, c, t, theta): return self._p2(abi.CRX, c, t, theta, "CRX")
    def cry(self, c, t, theta): return self._p2(abi.CRY, c, t, theta, "CRY")
    def crz(self, c, t, theta): return self._p2(abi.CRZ, c, t, theta, "CRZ")
    def cphase_param(self, c, t, theta): return self._p2(abi.CPHASE_PARAM, c, t, theta, "CP")
    def rxx(self, a, b, theta, textbook=False):
        return self._p2(abi.RXX, a, b, theta, "RXX", abi.FLAG_TEXTBOOK if textbook else 0)
    def ryy(self, a, b, theta, textbook=False):
        return self._p2(abi.RYY, a, b, theta, "RYY", abi.FLAG_TEXTBOOK if textbook else 0)
    def rzz(self, a, b, theta): return self._p2(abi.RZZ, a, b, theta, "RZZ")

    # bound-parameter builders used by ansatz templates: angle = theta[p]*scale + offset
    def ry_param(self, q, p, scale=1.0, offset=0.0):
        return self._p1(abi.RY, q, [offset], "RY", params=[p], scales=[scale])

    def rz_param(self, q, p, scale=1.0, offset=0.0):
        return self._p1(abi.RZ, q, [offset], "RZ", params=[p], scales=[scale])

    def rx_param(self, q, p, scale=1.0, offset=0.0):
        return self._p1(abi.RX, q, [offset], "RX", params=[p], scales=[scale])

    # -- composition (src/circuits/mod.rs:298-335) -------------------------
    def compose(self, other: "Circuit") -> "Circuit":
        if self._n != other._n:
            raise LogosQError(abi.LQ_ERR_QUBIT_MISMATCH,
                              f"Circuit qubit count mismatch: circuit has {self._n}, "
                              f"state has {other._n}")
        self._ops.extend(other._ops)
        self._packed = None
        return self

    def clone(self) -> "Circuit":
        """Circuit::clone: a copy whose operation list is independent."""
        c = Circuit(self._n)
        c._ops = list(self._ops)
        c._name = self._name
        return c

    def reversed(self) -> "Circuit":
        c = Circuit(self._n)
        for op in reversed(self._ops):
            c._ops.append(Operation(op.desc, op.qubits(), f"reversed_{op.name()}", op.dense))
        if self._name:
            c._name = f"{self._name}_reversed"
        return c

    # -- packed form --------------------------------------------------------
    def segments(self):
        """Split into runs of descriptors separated by dense full-state ops."""
        segs, cur = [], []
        for op in self._ops:
            if op.dense is not None:
                if cur:
                    segs.append(("desc", np.concatenate(cur)))
                    cur = []
                segs.append(("dense", op.dense))
            else:
                cur.append(op.desc)
        if cur:
            segs.append(("desc", np.concatenate(cur)))
        return segs

    def packed(self) -> np.ndarray:
        """All descriptors as one C-layout array (error if a dense op is present)."""
        if self._packed is None:
            if any(op.dense is not None for op in self._ops):
                raise LogosQError(abi.LQ_ERR_UNSUPPORTED,
                                  "circuit holds full-state matrix gates")
            self._packed = (np.concatenate([op.desc for op in self._ops])
                            if self._ops else abi.empty_gates(0))
        return self._packed

    # -- execution (src/circuits/mod.rs:196-375) --------------------------
    def add_noise(self, noise_model) -> "Circuit":
        """Circuit::add_noise (src/circuits/mod.rs:340-343)."""
        self._noise.append(noise_model)
        return self

    def _check_state(self, state):
        if state.num_qubits() != self._n:
            raise LogosQError(abi.LQ_ERR_QUBIT_MISMATCH,
                              f"Circuit qubit count mismatch: circuit has {self._n}, "
                              f"state has {state.num_qubits()}")

    def execute_without_noise(self, state, theta=None, mode: int = abi.EXEC_FUSED) -> None:
        """Circuit::execute_without_noise (src/circuits/mod.rs:196-209), one
        fused launch sequence for the whole circuit."""
        self._check_state(state)
        th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
        nth = 0 if th is None else len(th)
        thp = None if th is None else abi.f64_ptr(th)
        for kind, seg in self.segments():
            if kind == "dense":
                MatrixGate(seg).apply(state)
            else:
                call("lq_apply_circuit", state.handle, self._n, abi.gate_ptr(seg), len(seg),
                     thp, nth, mode)

    def execute(self, state, theta=None, mode: int = abi.EXEC_FUSED) -> None:
        """Circuit::execute (src/circuits/mod.rs:352-375): without noise models
        the whole circuit runs fused; with them, every gate is followed by every
        noise model, in order."""
        if not self._noise:
            return self.execute_without_noise(state, theta, mode)
        self._check_state(state)
        th = None if theta is None else np.ascontiguousarray(theta, dtype=np.float64)
        nth = 0 if th is None else len(th)
        thp = None if th is None else abi.f64_ptr(th)
        for op in self._ops:
            if op.dense is not None:
                MatrixGate(op.dense).apply(state)
            else:
                call("lq_apply_circuit", state.handle, self._n, abi.gate_ptr(op.desc), 1, thp,
                     nth, abi.EXEC_PER_GATE)
            for model in self._noise:
                model.apply(state)

    def last_stats(self, state):
        launches, passes = C.c_int(), C.c_int()
        call("lq_last_circuit_stats", state.handle, C.byref(launches), C.byref(passes))
        return launches.value, passes.value

    def expectation(self, observable: Gate) -> float:
        """Circuit::expectation (src/circuits/mod.rs:256-287): <psi|O psi> with
        O applied as a gate to a copy of the executed state."""
        from .states import State
        st = State.zero_state(self._n)
        self.execute(st)
        ob = st.clone()
        observable.apply(ob)
        return st.inner_product(ob).real

    def execute_and_measure(self, seed: int = 0):
        """execute_and_measure (src/circuits/mod.rs:216-233): measure_qubit(i)
        on a copy of the final state for every i."""
        from .states import State
        st = State.zero_state(self._n)
        self.execute(st)
        out = []
        for i in range(self._n):
            c = st.clone()
            out.append(c.measure_qubit(i, seed=seed + i))
            c.close()
        return out

    def execute_and_measure_with_noise(self, seed: int = 0):
        """execute_and_measure_with_noise (src/circuits/mod.rs:376-411): the same
        steps as execute_and_measure -- execute already applies the circuit's
        noise models after every gate."""
        return self.execute_and_measure(seed)

    def __repr__(self):
        # Debug for Circuit (src/circuits/mod.rs:597-608)
        lines = [f"Circuit: {self._name or 'Unnamed Circuit'} ({self._n} qubits)"]
        lines += [f"{i}: {op!r}" for i, op in enumerate(self._ops)]
        return "\n".join(lines) + "\n"

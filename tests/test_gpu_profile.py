"""GPU: the launch profiler (lq_profile_enable / lq_profile_read) that the
benchmark's per-kernel figures come from.  Each public call is timed as one
bracket of its kernel class; a reduction that runs inside a gate (the norm
pass of a renormalising gate) is counted toward the gate, not twice."""
import ctypes as C

import numpy as np
import pytest

from logosq_b200 import State, abi
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu

FUSED, GATE, REDUCE = 0, 1, 2


def read(cls):
    ms, cnt = C.c_double(), C.c_longlong()
    call("lq_profile_read", cls, C.byref(ms), C.byref(cnt))
    return ms.value, cnt.value


def one_gate(kind, qs, angles=(), flags=0, m=None):
    g = abi.empty_gates(1)
    g[0]["kind"] = kind
    g[0]["flags"] = flags
    for i, q in enumerate(qs):
        g[0]["q"][i] = q
    for i, a in enumerate(angles):
        g[0]["angle"][i] = a
    if m is not None:
        g[0]["m"][:len(m)] = m
    return g


def test_profile_counts_per_class_and_nesting():
    n = 14
    st = State.plus_state(n)
    other = State.plus_state(n)
    try:
        u3 = one_gate(abi.U3, [3], (0.3, 0.2, 0.1))
        h = np.array([1, 0, 1, 0, 1, 0, -1, 0], dtype=np.float64) / np.sqrt(2.0)
        hren = one_gate(abi.MATRIX1, [5], flags=abi.FLAG_RENORM, m=h)
        st.synchronize()
        call("lq_profile_enable", 1)
        for _ in range(2):
            call("lq_apply_gate", st.handle, abi.gate_ptr(u3), None, 0)
        # a renormalising gate: the gate sweep, then the norm and scale passes
        call("lq_apply_gate", st.handle, abi.gate_ptr(hren), None, 0)
        st.synchronize()
        ms_g, cnt_g = read(GATE)
        assert cnt_g == 3 and ms_g > 0.0
        assert read(REDUCE)[1] == 0  # the nested norm pass counts toward its gate

        out = C.c_double()
        term = np.zeros(1, dtype=abi.TERM_DTYPE)
        term[0]["coefficient"] = 1.0
        term[0]["zmask"] = 1
        call("lq_expectation_pauli", st.handle, abi.term_ptr(term), 1, abi.Y_REFERENCE,
             C.byref(out), None)
        call("lq_norm_sqr", st.handle, C.byref(out))
        assert abs(out.value - 1.0) < 1e-12
        o2 = (C.c_double * 2)()
        call("lq_inner_product", st.handle, other.handle, o2)
        ms_r, cnt_r = read(REDUCE)
        assert cnt_r == 3 and ms_r > 0.0
        assert read(GATE)[1] == 3

        g = np.concatenate([one_gate(abi.H, [q]) for q in range(n)])
        call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, abi.EXEC_FUSED)
        st.synchronize()
        passes = C.c_int()
        call("lq_last_circuit_stats", st.handle, None, C.byref(passes))
        assert passes.value >= 1 and read(FUSED)[1] == passes.value

        # enabling again resets every counter
        call("lq_profile_enable", 1)
        assert all(read(c) == (0.0, 0) for c in range(5))
    finally:
        call("lq_profile_enable", 0)
        st.close()
        other.close()


def test_profile_off_records_nothing():
    st = State.plus_state(10)
    try:
        call("lq_profile_enable", 0)
        u3 = one_gate(abi.U3, [2], (0.3, 0.2, 0.1))
        call("lq_apply_gate", st.handle, abi.gate_ptr(u3), None, 0)
        st.synchronize()
        assert read(GATE) == (0.0, 0)
    finally:
        st.close()


def test_profile_rejects_unknown_class():
    from logosq_b200 import LogosQError
    with pytest.raises(LogosQError):
        call("lq_profile_read", 5, None, None)

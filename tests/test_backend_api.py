"""CPU: the QuantumStateBackend methods of State (src/states/backend.rs:14-60,
src/states/mod.rs:394-486) call the engine's entry points with the right
arguments: checked with a recording stand-in for the C calls, so no GPU is
needed (the entry points themselves are covered by the GPU parity tests)."""
import ctypes as C

import numpy as np
import pytest

from logosq_b200 import LogosQError, State, abi, gates, states


class Rec:
    def __init__(self):
        self.calls = []

    def __call__(self, name, *args):
        if name in ("lq_apply_matrix1", "lq_apply_matrix2"):
            k = 8 if name == "lq_apply_matrix1" else 32
            buf = np.ctypeslib.as_array(args[-1], shape=(k,)).copy()
            self.calls.append((name, tuple(int(a) for a in args[1:-1]), buf))
        elif name == "lq_apply_dense":
            dim = args[2].value
            buf = np.ctypeslib.as_array(args[1], shape=(2 * dim * dim,)).copy()
            self.calls.append((name, (dim,), buf))
        else:
            self.calls.append((name, (), None))


@pytest.fixture
def fake(monkeypatch):
    rec = Rec()
    monkeypatch.setattr(states, "call", rec)
    monkeypatch.setattr(gates, "call", rec)
    st = State.__new__(State)
    st._n, st._h, st._dtype = 3, C.c_void_p(1), abi.LQ_C128
    st.close = lambda: None  # the stand-in owns no device state
    yield st, rec
    st._h = None


def interleaved(m):
    return np.ascontiguousarray(m, dtype=np.complex128).view(np.float64).reshape(-1)


def test_single_qubit_matrix(fake):
    st, rec = fake
    m = gates.ry_matrix(0.7)
    st.apply_single_qubit_matrix(2, m)
    assert [c[0] for c in rec.calls] == ["lq_apply_matrix1", "lq_normalize"]
    assert rec.calls[0][1] == (2,) and np.array_equal(rec.calls[0][2], interleaved(m))


def test_two_qubit_matrix_control_is_high_bit(fake):
    st, rec = fake
    m = gates.cnot_matrix()
    st.apply_two_qubit_matrix(0, 2, m)
    assert [c[0] for c in rec.calls] == ["lq_apply_matrix2", "lq_normalize"]
    assert rec.calls[0][1] == (0, 2) and np.array_equal(rec.calls[0][2], interleaved(m))


def test_three_qubit_and_full_matrix_use_the_dense_path(fake):
    st, rec = fake
    m = gates.toffoli_matrix()
    st.apply_three_qubit_matrix(0, 1, 2, m)
    st.apply_full_matrix(m)
    assert [c[0] for c in rec.calls] == ["lq_apply_dense", "lq_apply_dense"]
    assert rec.calls[0][1] == (8,) and np.array_equal(rec.calls[0][2], interleaved(m))


def test_errors(fake):
    st, rec = fake
    with pytest.raises(LogosQError, match=r"Invalid qubit index: 3 \(must be < 3\)"):
        st.apply_single_qubit_matrix(3, np.eye(2))
    with pytest.raises(LogosQError):
        st.apply_two_qubit_matrix(0, 5, np.eye(4))
    with pytest.raises(LogosQError):
        st.apply_single_qubit_matrix(0, np.eye(4))
    with pytest.raises(LogosQError):
        st.apply_full_matrix(np.eye(4))  # 2 qubits' matrix on a 3-qubit state
    assert rec.calls == []

"""GPU: precision form (complex64 state, 5-qubit blocks on tcgen05 with 3xTF32)
against the complex128 engine on the same circuit.

Bars, relative to the state's RMS amplitude (amplitudes are O(2^-n/2), so an
absolute bar would be loose for large n): one block 1e-5 of the largest
amplitude (plain TF32 products give ~1e-3: tests/test_tc_split_emulation.py);
whole circuits max-abs 1e-5 x RMS, |1 - fidelity| 1e-8 and the FP64 norm of
the input kept to 1e-8 (rounding the restored amplitudes to complex64 moves the
norm by ~1e-9, so the unnormalised fidelity cannot be held tighter).  Measured
on a B200: 1.1-5.8e-6 x RMS (12-20 qubits,
up to 20 layers), norm within 1e-10 -- the tensor cores' FP32 accumulation
shrinks the state by ~6e-7 per block, which the engine removes by restoring
the input's FP64 norm after the circuit."""
import ctypes as C

import numpy as np
import pytest

from logosq_b200 import State, abi, workloads
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu


def run_c128(n, g, v=None):
    st = State.zero_state(n)
    if v is not None:
        st.set_vector(v)
    call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, abi.EXEC_FUSED)
    out = st.vector()
    st.close()
    return out


def run_tc(n, g, v=None):
    st = State.zero_state(n, dtype=abi.LQ_C64)
    if v is not None:
        st.set_vector(v)
    nb, npass = C.c_int(), C.c_int()
    call("lq_apply_circuit_tc", st.handle, n, abi.gate_ptr(g), len(g), None, 0, C.byref(nb),
         C.byref(npass))
    out = st.vector()
    norm = st.norm_sqr()
    st.close()
    return out, norm, nb.value, npass.value


def test_tc_single_block_is_3xtf32_accurate():
    """One 5-qubit block (U3 on five qubits): relative error ~1e-7, far below
    the ~1e-3 of single TF32 products."""
    n = 12
    v = workloads.gaussian_state(n, 9).astype(np.complex64).astype(np.complex128)
    g = workloads.brickwork_u3(n, 1, seed=4)[:5]  # U3 on qubits 0..4: one block
    want = run_c128(n, g, v)
    got, _, nb, _ = run_tc(n, g, v)
    assert nb == 1
    rel = np.abs(got - want).max() / np.abs(want).max()
    assert rel < 1e-5, rel


@pytest.mark.parametrize("n,layers", [(12, 4), (14, 6), (17, 8)])
def test_tc_brickwork_matches_complex128(n, layers):
    g = workloads.brickwork_u3(n, layers, seed=3)
    want = run_c128(n, g)
    got, norm, nb, npass = run_tc(n, g)
    assert nb > 0 and npass > 0
    rms = np.sqrt(np.mean(np.abs(want) ** 2))
    err = np.abs(got - want).max() / rms
    fid = abs(np.vdot(want, got)) ** 2
    assert err < 1e-5, err
    assert abs(fid - 1) < 1e-8, fid
    assert abs(norm - 1) < 1e-8, norm


def test_tc_qft_random_state():
    n = 14
    v = workloads.gaussian_state(n, 5)
    g = workloads.qft_gates(n)
    want = run_c128(n, g, v)
    got, norm, _, _ = run_tc(n, g, v)
    rms = np.sqrt(np.mean(np.abs(want) ** 2))
    assert np.abs(got - want).max() / rms < 1e-5
    assert abs(abs(np.vdot(want, got)) ** 2 - 1) < 1e-8
    assert abs(norm - 1) < 1e-8


def test_tc_rejects_complex128_state():
    st = State.zero_state(12)
    g = workloads.brickwork_u3(12, 1, seed=1)
    from logosq_b200 import LogosQError
    with pytest.raises(LogosQError) as e:
        call("lq_apply_circuit_tc", st.handle, 12, abi.gate_ptr(g), len(g), None, 0, None, None)
    assert e.value.code == abi.LQ_ERR_UNSUPPORTED

"""Parity of the headline circuit at its own size: the 28-qubit, 20-layer random
U3 + CNOT brickwork (seed 2, from |0...0>) through the fused Circuit::execute
path, against the oracle's restatement of the reference loops.

The reference generator is rqc::generate_supremacy_circuit
(src/algorithms/rqc.rs:236-268) with U3 in place of RZ-RY-RZ; the overlap is
State::inner_product_parallel (src/states/mod.rs:350-365).  The oracle runs in
threaded mode, which is bitwise identical to its faithful (reference-serial)
mode.  Every tile width the autotuner may pick (10, 11, 12) runs the same
circuit, so pair folding, the window planner and both register forms of the
fused kernel are covered at this size.

Bars: max-abs 1e-12 per amplitude, |1 - fidelity| 1e-12.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from logosq_b200 import State, abi, workloads
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu
N, LAYERS, SEED = 28, 20, 2
TOL = 1e-12


@pytest.fixture(scope="module")
def want():
    g = workloads.brickwork_u3(N, LAYERS, seed=SEED)
    oracle.set_threads(oracle.max_threads())
    try:
        v = oracle.apply_circuit(oracle.zero_state(N), g)
    finally:
        oracle.set_threads(1)
    return v


@pytest.mark.parametrize("tile_bits", [10, 11, 12])
def test_brickwork_28q_20_layers_vs_oracle(want, tile_bits):
    g = workloads.brickwork_u3(N, LAYERS, seed=SEED)
    old = C.c_int()
    call("lq_get_fusion_width", C.byref(old))
    call("lq_set_fusion_width", tile_bits)
    st = State.zero_state(N)
    try:
        call("lq_apply_circuit", st.handle, N, abi.gate_ptr(g), len(g), None, 0, abi.EXEC_FUSED)
        got = st.vector()
    finally:
        st.close()
        call("lq_set_fusion_width", old.value)
    max_abs = float(np.abs(got - want).max())
    fid = abs(np.vdot(want, got)) ** 2
    assert max_abs < TOL, (tile_bits, max_abs)
    assert abs(fid - 1.0) < TOL, (tile_bits, fid)

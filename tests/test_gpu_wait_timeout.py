"""GPU: the give-up path of a bounded device wait, made to run out on purpose
without faulting, trapping or hanging anything.

lq_check_wait_timeout queues a kernel that waits on a shared-memory barrier
nothing completes and gives up after a short, caller-given number of polls --
the same exit every pipeline wait of the fused and tensor-core passes takes
after its own bound.  The next lq_state_synchronize must report
LQ_ERR_TIMEOUT (the reference's error surface is LogosQError,
src/error.rs:9-64), and the handle and CUDA context must stay usable: the
following circuit runs and matches the oracle, and synchronising again
succeeds."""
import numpy as np
import pytest

import oracle
from logosq_b200 import LogosQError, State, abi, workloads
from logosq_b200._lib import call

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("polls", [1, 4096])
def test_wait_runs_out_and_handle_stays_usable(polls):
    n = 12
    st = State.zero_state(n)
    try:
        call("lq_check_wait_timeout", st.handle, polls)
        with pytest.raises(LogosQError) as e:
            st.synchronize()
        assert e.value.code == abi.LQ_ERR_TIMEOUT
        # the condition is cleared once reported
        st.synchronize()
        g = workloads.brickwork_u3(n, 3, seed=11)
        call("lq_apply_circuit", st.handle, n, abi.gate_ptr(g), len(g), None, 0, abi.EXEC_FUSED)
        st.synchronize()
        want = oracle.apply_circuit(oracle.zero_state(n), g)
        assert np.abs(st.vector() - want).max() < 1e-12
    finally:
        st.close()


def test_poll_bound_is_checked():
    st = State.zero_state(5)
    try:
        for bad in (0, (1 << 20) + 1):
            with pytest.raises(LogosQError) as e:
                call("lq_check_wait_timeout", st.handle, bad)
            assert e.value.code == abi.LQ_ERR_INVALID_ARG
        st.synchronize()
    finally:
        st.close()

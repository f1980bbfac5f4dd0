"""GPU: the allocation-free Pauli-sum expectation (lq_expectation_pauli_static).

Some callers cannot call cudaMalloc -- their device memory belongs to a host
framework's own allocator or budget, or they must not put the device-wide
synchronisation of an allocation into the middle of their stream work.  This
entry point keeps its scratch in a fixed array inside the library and works on
caller-owned device memory; here it must give the same energy as the regular
lq_expectation_pauli on two calls in a row (the second call finds the first
call's leftovers in the shared scratch array).  Collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from logosq_b200 import State, abi, workloads
from logosq_b200._lib import LogosQError, call

pytestmark = pytest.mark.gpu


def _terms(n, count, seed):
    rng = workloads.SplitMix64(seed)
    t = np.zeros(count, dtype=abi.TERM_DTYPE)
    for k in range(count):
        x = rng.randint(0, (1 << n) - 1) if k % 3 else 0
        z = rng.randint(0, (1 << n) - 1)
        t[k]["coefficient"] = rng.uniform(-1, 1)
        t[k]["xmask"] = x
        t[k]["zmask"] = z
        t[k]["ny"] = bin(x & z).count("1")
    return t


def _regular(st, terms, yconv):
    out = C.c_double()
    call("lq_expectation_pauli", st.handle, abi.term_ptr(terms), len(terms), yconv, C.byref(out),
         None)
    return out.value


def _static(st, terms, yconv, dtype=abi.LQ_C128):
    ptr, stream = C.c_void_p(), C.c_void_p()
    call("lq_state_device_ptr", st.handle, C.byref(ptr))
    call("lq_state_stream", st.handle, C.byref(stream))
    out = C.c_double()
    call("lq_expectation_pauli_static", ptr, st.num_qubits(), dtype, abi.term_ptr(terms),
         len(terms), yconv, stream, C.byref(out))
    return out.value


def test_static_expectation_matches_regular_two_calls():
    cases = [(15, 60, 1, abi.Y_REFERENCE), (12, 300, 2, abi.Y_TEXTBOOK)]
    for n, count, seed, yconv in cases:  # two calls in a row, different inputs
        st = State.zero_state(n)
        st.set_vector(workloads.gaussian_state(n, seed))
        terms = _terms(n, count, seed)
        want = _regular(st, terms, yconv)
        got = _static(st, terms, yconv)
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (n, got, want)
        st.close()


def test_static_expectation_rejects_too_many_terms():
    st = State.zero_state(4)
    terms = _terms(4, 1025, 3)
    with pytest.raises(LogosQError) as e:
        _static(st, terms, abi.Y_REFERENCE)
    assert e.value.code == abi.LQ_ERR_UNSUPPORTED


def test_static_expectation_matches_oracle():
    """Against the oracle's restatement of PauliTerm::expectation
    (src/optimization/observable.rs:95-147), not only against the engine:
    X-mask-0 terms and X-mask groups, both Y conventions, small and large n,
    and exactly the 1024-term limit."""
    import oracle
    for n, count, seed, yconv in [(2, 12, 5, abi.Y_REFERENCE), (13, 200, 6, abi.Y_TEXTBOOK),
                                  (16, 1024, 7, abi.Y_REFERENCE)]:
        v = workloads.gaussian_state(n, seed)
        terms = _terms(n, count, seed)
        st = State.zero_state(n)
        try:
            st.set_vector(v)
            got = _static(st, terms, yconv)
        finally:
            st.close()
        want = oracle.expectation(v, terms, yconv)
        assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (n, count, got, want)


def test_static_expectation_complex64_state():
    """A complex64 state (the precision form's storage): same value as the
    regular entry point on the same state, within FP64-accumulation noise."""
    n = 14
    st = State.zero_state(n, dtype=abi.LQ_C64)
    try:
        st.set_vector(workloads.gaussian_state(n, 3))
        terms = _terms(n, 90, 4)
        want = _regular(st, terms, abi.Y_REFERENCE)
        got = _static(st, terms, abi.Y_REFERENCE, dtype=abi.LQ_C64)
    finally:
        st.close()
    assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (got, want)


def test_static_expectation_rejects_host_pointer():
    """A host buffer is not device memory: refused before any kernel runs."""
    buf = np.zeros(2 * 16, dtype=np.float64)
    out = C.c_double()
    terms = _terms(4, 3, 1)
    with pytest.raises(LogosQError) as e:
        call("lq_expectation_pauli_static", buf.ctypes.data_as(C.c_void_p), 4, abi.LQ_C128,
             abi.term_ptr(terms), len(terms), abi.Y_REFERENCE, None, C.byref(out))
    assert e.value.code == abi.LQ_ERR_INVALID_ARG


def test_static_refuses_a_capturing_stream():
    """The call copies its term table from host stack memory and waits for its
    stream, so it must refuse a stream that is being captured into a graph
    (and leave the capture intact)."""
    import torch
    n = 10
    st = State.plus_state(n)
    try:
        ptr = C.c_void_p()
        call("lq_state_device_ptr", st.handle, C.byref(ptr))
        terms = _terms(n, 8, 5)
        want = _regular(st, terms, abi.Y_REFERENCE)
        s = torch.cuda.Stream()
        x = torch.zeros(4, device="cuda")
        g = torch.cuda.CUDAGraph()
        out = C.c_double()
        with torch.cuda.graph(g, stream=s):
            x.add_(1.0)
            with pytest.raises(LogosQError) as e:
                call("lq_expectation_pauli_static", ptr, n, abi.LQ_C128, abi.term_ptr(terms),
                     len(terms), abi.Y_REFERENCE, C.c_void_p(s.cuda_stream), C.byref(out))
        assert e.value.code == abi.LQ_ERR_UNSUPPORTED
        g.replay()
        torch.cuda.synchronize()
        assert float(x[0]) == 1.0
        del g
        # outside the capture the same call works
        assert abs(_static(st, terms, abi.Y_REFERENCE) - want) < 1e-12 * max(1, abs(want))
    finally:
        st.close()

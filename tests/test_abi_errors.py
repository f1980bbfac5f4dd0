"""CPU: the C ABI's argument checks, which run on the host before any CUDA call
(so they are testable without a GPU).  The error kinds mirror LogosQError
(src/error.rs:9-61): a bad qubit count is InvalidStateDimension, a wrong
parameter count ParameterCountMismatch; a NULL handle or output pointer is
LQ_ERR_INVALID_ARG, and destroying a NULL handle is a no-op like free(NULL)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from logosq_b200 import _lib, abi

ROOT = Path(__file__).resolve().parent.parent
HEADER = (ROOT / "include" / "logosq_b200.h").read_text()


def raw():
    return _lib.lib()


def handle_entry_points():
    """(name, number of parameters) of every declared entry point whose first
    parameter is a state, batch or network handle."""
    out = []
    for name, params in re.findall(r"^\s*int\s+(lq_\w+)\s*\(([^;]*?)\);", HEADER,
                                   flags=re.M | re.S):
        ps = [p.strip() for p in params.replace("\n", " ").split(",") if p.strip()]
        if ps and re.search(r"\b(lq_state|lq_batch|lq_mlp)\s*\*\s*\w+$", ps[0]):
            out.append((name, len(ps)))
    return out


def call_null(name, nparams):
    f = getattr(raw(), name)
    f.restype = C.c_int
    f.argtypes = [C.c_void_p] * nparams
    return f(*([None] * nparams))


def last_error():
    return raw().lq_last_error().decode()


def test_header_has_handle_entry_points():
    names = [n for n, _ in handle_entry_points()]
    for must in ("lq_apply_gate", "lq_expectation_pauli", "lq_batch_gradients",
                 "lq_mlp_forward", "lq_noise_pauli", "lq_state_destroy"):
        assert must in names


@pytest.mark.parametrize("name,nparams", handle_entry_points(), ids=lambda x: str(x))
def test_null_handle_is_rejected(name, nparams):
    rc = call_null(name, nparams)
    if name.endswith("_destroy"):
        assert rc == abi.LQ_OK
    else:
        assert rc == abi.LQ_ERR_INVALID_ARG, (name, rc, last_error())
        assert last_error()


@pytest.mark.parametrize("n", [-1, 0, 37, 64])
def test_state_create_rejects_bad_qubit_count(n):
    out = C.c_void_p()
    assert raw().lq_state_create(n, abi.LQ_C128, C.byref(out)) == abi.LQ_ERR_STATE_DIMENSION
    assert "Invalid state dimension" in last_error()
    assert not out.value


def test_state_create_rejects_bad_dtype_and_null_output():
    out = C.c_void_p()
    assert raw().lq_state_create(3, 7, C.byref(out)) == abi.LQ_ERR_INVALID_ARG
    assert raw().lq_state_create(3, abi.LQ_C128, None) == abi.LQ_ERR_INVALID_ARG


def test_fusion_width_range():
    w0 = C.c_int()
    assert raw().lq_get_fusion_width(C.byref(w0)) == abi.LQ_OK
    try:
        for bad in (0, 4, 13):
            assert raw().lq_set_fusion_width(bad) == abi.LQ_ERR_INVALID_ARG
        for good in (5, 10, 12):
            assert raw().lq_set_fusion_width(good) == abi.LQ_OK
            w = C.c_int()
            raw().lq_get_fusion_width(C.byref(w))
            assert w.value == good
    finally:
        raw().lq_set_fusion_width(w0.value)


@pytest.mark.parametrize("cls", [-1, 5])
def test_profile_read_rejects_unknown_class(cls):
    assert raw().lq_profile_read(cls, None, None) == abi.LQ_ERR_INVALID_ARG


def test_static_expectation_checks_arguments():
    """The allocation-free expectation refuses bad arguments before touching the
    device: NULL pointers, an unknown dtype, and more terms than its fixed
    scratch holds (1024)."""
    f = raw().lq_expectation_pauli_static
    terms = (abi.LqPauliTerm * 1025)()
    out = C.c_double()
    fake = C.c_void_p(256)  # never dereferenced: every case fails its host-side check
    assert f(None, 4, abi.LQ_C128, terms, 1, 0, None, C.byref(out)) == abi.LQ_ERR_INVALID_ARG
    assert f(fake, 4, abi.LQ_C128, terms, 1, 0, None, None) == abi.LQ_ERR_INVALID_ARG
    assert f(fake, 4, 9, terms, 1, 0, None, C.byref(out)) == abi.LQ_ERR_INVALID_ARG
    assert f(fake, 4, abi.LQ_C128, terms, 1025, 0, None, C.byref(out)) == abi.LQ_ERR_UNSUPPORTED
    assert "1024" in last_error()


def test_constructors_reject_bad_shapes():
    out = C.c_void_p()
    assert raw().lq_mlp_create(0, 256, 3, 128, 1, C.byref(out)) == abi.LQ_ERR_INVALID_ARG
    assert raw().lq_batch_create(None, 0, C.byref(out)) == abi.LQ_ERR_INVALID_ARG


def test_python_mirror_raises_logosq_error():
    with pytest.raises(_lib.LogosQError) as ei:
        _lib.call("lq_set_fusion_width", 99)
    assert ei.value.code == abi.LQ_ERR_INVALID_ARG

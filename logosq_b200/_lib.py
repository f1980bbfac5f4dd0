"""Loader for liblogosq_b200.so with the C prototypes of include/logosq_b200.h.

The engine has no CPU fallback: if the library is missing or no CUDA device is
visible, every call that needs the device raises LogosQError.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

from . import abi

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("LOGOSQ_B200_LIB", _HERE / "liblogosq_b200.so"))

_lib = None


class LogosQError(RuntimeError):
    """A non-zero status from the engine (mirrors LogosQError, src/error.rs:9-61)."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.kind = abi.STATUS_NAMES.get(code, f"Status{code}")
        super().__init__(f"{self.kind}: {message}")


_P = C.c_void_p
_PD = C.POINTER(C.c_double)
_PF = C.POINTER(C.c_float)
_PI = C.POINTER(C.c_int)
_PG = C.POINTER(abi.LqGate)
_PT = C.POINTER(abi.LqPauliTerm)

_PROTOS = {
    "lq_last_error": (C.c_char_p, []),
    "lq_version": (C.c_int, []),
    "lq_device_count": (C.c_int, [_PI]),
    "lq_set_device": (C.c_int, [C.c_int]),
    "lq_set_alloc_limit": (C.c_int, [C.c_uint64]),
    "lq_profile_enable": (C.c_int, [C.c_int]),
    "lq_profile_read": (C.c_int, [C.c_int, _PD, C.POINTER(C.c_longlong)]),
    "lq_state_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(_P)]),
    "lq_state_destroy": (C.c_int, [_P]),
    "lq_state_num_qubits": (C.c_int, [_P, _PI]),
    "lq_state_dtype": (C.c_int, [_P, _PI]),
    "lq_state_set_basis": (C.c_int, [_P, C.c_uint64]),
    "lq_state_set_plus": (C.c_int, [_P]),
    "lq_state_upload": (C.c_int, [_P, _PD, C.c_size_t]),
    "lq_state_download": (C.c_int, [_P, _PD, C.c_size_t]),
    "lq_state_upload_c64": (C.c_int, [_P, _PF, C.c_size_t]),
    "lq_state_download_c64": (C.c_int, [_P, _PF, C.c_size_t]),
    "lq_state_copy": (C.c_int, [_P, _P]),
    "lq_state_tensor_product": (C.c_int, [_P, _P, _P]),
    "lq_apply_dense": (C.c_int, [_P, _PD, C.c_uint64]),
    "lq_state_synchronize": (C.c_int, [_P]),
    "lq_check_wait_timeout": (C.c_int, [_P, C.c_uint]),
    "lq_state_device_ptr": (C.c_int, [_P, C.POINTER(_P)]),
    "lq_state_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "lq_norm_sqr": (C.c_int, [_P, _PD]),
    "lq_normalize": (C.c_int, [_P]),
    "lq_probabilities": (C.c_int, [_P, _PD, C.c_size_t]),
    "lq_probability": (C.c_int, [_P, C.c_uint64, _PD]),
    "lq_inner_product": (C.c_int, [_P, _P, _PD]),
    "lq_measure_shots": (C.c_int, [_P, C.c_uint64, C.c_uint64, C.POINTER(C.c_uint64)]),
    "lq_expectation_pauli": (C.c_int, [_P, _PT, C.c_int, C.c_int, _PD, _PD]),
    "lq_expectation_pauli_static": (C.c_int, [_P, C.c_int, C.c_int, _PT, C.c_int, C.c_int, _P,
                                              _PD]),
    "lq_apply_gate": (C.c_int, [_P, _PG, _PD, C.c_int]),
    "lq_apply_matrix1": (C.c_int, [_P, C.c_int, _PD]),
    "lq_apply_controlled1": (C.c_int, [_P, C.c_int, C.c_int, _PD]),
    "lq_apply_diagonal": (C.c_int, [_P, C.c_int, _PI, _PD]),
    "lq_apply_swap": (C.c_int, [_P, C.c_int, C.c_int]),
    "lq_apply_matrix2": (C.c_int, [_P, C.c_int, C.c_int, _PD]),
    "lq_apply_block": (C.c_int, [_P, C.c_int, _PI, _PD]),
    "lq_apply_circuit": (C.c_int, [_P, C.c_int, _PG, C.c_int, _PD, C.c_int, C.c_int]),
    "lq_last_circuit_stats": (C.c_int, [_P, _PI, _PI]),
    "lq_apply_circuit_tc": (C.c_int, [_P, C.c_int, _PG, C.c_int, _PD, C.c_int, _PI, _PI]),
    "lq_plan_circuit": (C.c_int, [C.c_int, _PG, C.c_int, _PI, _PI, _PI]),
    "lq_set_fusion_width": (C.c_int, [C.c_int]),
    "lq_get_fusion_width": (C.c_int, [_PI]),
    "lq_plan_dump": (C.c_int, [C.c_int, _PG, C.c_int, _PD, C.c_int, _P, C.c_size_t,
                               C.POINTER(C.c_size_t)]),
    "lq_ansatz_energy": (C.c_int, [_P, _PG, C.c_int, _PD, C.c_int, _PT, C.c_int, C.c_int, _PD]),
    "lq_parameter_shift": (
        C.c_int, [_P, _PG, C.c_int, _PD, C.c_int, _PT, C.c_int, C.c_int, C.c_double, _PD]),
    "lq_finite_difference": (
        C.c_int, [_P, _PG, C.c_int, _PD, C.c_int, _PT, C.c_int, C.c_int, C.c_double, _PD]),
    "lq_batch_create": (C.c_int, [C.POINTER(abi.LqVqeInstance), C.c_int, C.POINTER(_P)]),
    "lq_batch_destroy": (C.c_int, [_P]),
    "lq_batch_num_params": (C.c_int, [_P, _PI]),
    "lq_batch_gradients": (C.c_int, [_P, _PD, C.c_double, _PD, _PD]),
    "lq_batch_tuning": (C.c_int, [_P, _PI, _PI]),
    "lq_batch_prefix_info": (C.c_int, [_P, _PI, C.POINTER(C.c_uint64)]),
    "lq_batch_set_tile_bits": (C.c_int, [_P, C.c_int]),
    "lq_noise_pauli": (C.c_int, [_P, C.c_int, C.c_int]),
    "lq_noise_amplitude_damping": (C.c_int, [_P, C.c_double, _PI, C.c_int]),
    "lq_noise_phase_damping": (C.c_int, [_P, C.c_double, _PI, C.c_int]),
    "lq_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(_P)]),
    "lq_mlp_destroy": (C.c_int, [_P]),
    "lq_mlp_num_params": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "lq_mlp_get_params": (C.c_int, [_P, _PF, C.c_int64]),
    "lq_mlp_set_params": (C.c_int, [_P, _PF, C.c_int64]),
    "lq_mlp_get_grads": (C.c_int, [_P, _PF, C.c_int64]),
    "lq_mlp_forward": (C.c_int, [_P, _PF, C.c_int, _PF]),
    "lq_mlp_loss_grad": (C.c_int, [_P, _PF, _PF, _PF, C.c_int, _PD]),
    "lq_mlp_backward": (C.c_int, [_P, _PF, _PF, C.c_int]),
    "lq_mlp_adam_step": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, C.c_float]),
    "lq_mlp_reset_adam": (C.c_int, [_P]),
    "lq_lanczos_ground_energy": (C.c_int, [C.c_int, _PT, C.c_int, C.c_int, C.c_double, C.c_uint64,
                                           _PD, _PI]),
}


def exported_symbols() -> list[str]:
    return list(_PROTOS)


def lib():
    """The loaded engine library (raises LogosQError if it cannot be loaded)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise LogosQError(
                abi.LQ_ERR_UNSUPPORTED,
                f"{LIB_PATH} is not built; run `python -m logosq_b200.build` (there is no CPU "
                "fallback)")
        lb = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _PROTOS.items():
            fn = getattr(lb, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = lb
    return _lib


def check(rc: int) -> None:
    if rc != abi.LQ_OK:
        msg = lib().lq_last_error()
        raise LogosQError(rc, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def device_count() -> int:
    n = C.c_int(0)
    rc = lib().lq_device_count(C.byref(n))
    return n.value if rc == abi.LQ_OK else 0

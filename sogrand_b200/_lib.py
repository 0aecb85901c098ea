"""ctypes binding of libsogrand_b200.so (the C ABI in include/sogrand_b200.h).

The shared library is built in-tree by ``make -C sogrand_b200/csrc`` (or
``__graft_entry__.build()``).  There is no fallback: if the library is
missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsogrand_b200.so")

SG_N = 16
SG_K = 8
SG_CUBE = 4096
SG_INFO_BITS = 512
SG_INFO_BYTES = 64
SG_MAX_IMAX = 50
SG_MAX_PHASES = 3 * SG_MAX_IMAX
SG_MAX_L = 8

STATUS = {
    0: "SG_OK",
    1: "SG_ERR_ARG",
    2: "SG_ERR_CUDA",
    3: "SG_ERR_NONFINITE",
    4: "SG_ERR_IO",
    5: "SG_ERR_NOMEM",
    6: "SG_ERR_TIMEOUT",
}


class SgParams(C.Structure):
    _fields_ = [
        ("L", C.c_int32),
        ("Imax", C.c_int32),
        ("Tmax", C.c_uint64),
        ("thres", C.c_double),
        ("alpha", C.c_double * SG_MAX_PHASES),
    ]


class SgCwStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_double),
        ("ng", C.c_uint64),
        ("ng_p", C.c_uint64),
        ("converged", C.c_int32),
        ("phases", C.c_int32),
    ]


class SgRunSummary(C.Structure):
    _fields_ = [
        ("blocks", C.c_uint64),
        ("total_iterations", C.c_double),
        ("total_ng", C.c_uint64),
        ("total_ng_p", C.c_uint64),
        ("seconds", C.c_double),
    ]


class SgDecodeSummary(C.Structure):
    _fields_ = [
        ("blocks", C.c_uint64),
        ("converged", C.c_uint64),
        ("nonfinite", C.c_uint64),
        ("total_ng", C.c_uint64),
        ("total_ng_p", C.c_uint64),
        ("bits_compared", C.c_uint64),
        ("bit_errors", C.c_uint64),
        ("block_errors", C.c_uint64),
        ("total_iterations", C.c_double),
        ("timeouts", C.c_uint64),
        ("device_error", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


# every symbol include/sogrand_b200.h declares, with its signature
_VP = C.c_void_p
_SIGS = {
    "sg_params_default": (None, [C.POINTER(SgParams)]),
    "sg_decode_device": (C.c_int, [_VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, _VP]),
    "sg_decode_host": (C.c_int, [_VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP]),
    "sg_bitso_device": (C.c_int, [_VP, C.c_size_t, C.c_int32, C.c_uint64, C.c_double, _VP, _VP, _VP, _VP, _VP]),
    "sg_bitso_host": (C.c_int, [_VP, C.c_size_t, C.c_int32, C.c_uint64, C.c_double, _VP, _VP, _VP, _VP]),
    "sg_decode_file": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(SgParams), C.c_size_t, C.POINTER(SgRunSummary)]),
    "sg_decode_summary_device": (C.c_int, [_VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, _VP]),
    "sg_decode_summary_device_noalloc": (C.c_int, [_VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, _VP]),
    "sg_wilson_interval": (C.c_int, [C.c_uint64, C.c_uint64, C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]),
    "sg_channel_sigma": (C.c_double, [C.c_double]),
    "sg_gen_info_host": (C.c_int, [C.c_uint64, C.c_uint64, C.c_size_t, _VP]),
    "sg_encode_host": (C.c_int, [_VP, C.c_size_t, _VP]),
    "sg_gen_llr_host": (C.c_int, [C.c_uint64, C.c_uint64, C.c_size_t, C.c_double, C.c_double, C.c_double, _VP, _VP]),
    "sg_gen_llr_device": (
        C.c_int,
        [C.c_uint64, C.c_uint64, C.c_size_t, C.c_double, C.c_double, C.c_double, _VP, _VP, _VP],
    ),
    "sg_pattern_order": (C.c_size_t, [C.c_int32, _VP, C.c_size_t]),
    "sg_set_math_mode": (C.c_int, [C.c_int32]),
    "sg_get_math_mode": (C.c_int32, []),
    "sg_set_wait_limit": (C.c_int, [C.c_uint64]),
    "sg_get_wait_limit": (C.c_uint64, []),
    "sg_check_device": (C.c_int, [_VP]),
    "sg_guess_ceiling": (C.c_int, [C.c_ulonglong, C.c_int32, C.POINTER(C.c_double)]),
    "sg_forward_device": (C.c_int, [_VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, _VP, _VP]),
    "sg_backward_device": (C.c_int, [_VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, C.c_int32, _VP, _VP, _VP,
                                     _VP]),
    "sg_batch_create": (C.c_int, [C.POINTER(C.c_void_p)]),
    "sg_batch_destroy": (C.c_int, [_VP]),
    "sg_batch_decode": (C.c_int, [_VP, _VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, _VP]),
    "sg_batch_capture": (C.c_int, [_VP, _VP, C.c_size_t, C.POINTER(SgParams), _VP, _VP, _VP, _VP]),
    "sg_batch_replay": (C.c_int, [_VP, _VP]),
    "sg_batch_check": (C.c_int, [_VP]),
    "sg_batch_variant_count": (C.c_int, []),
    "sg_batch_variant_name": (C.c_char_p, [C.c_int]),
    "sg_batch_set_variant": (C.c_int, [C.c_int]),
    "sg_batch_get_variant": (C.c_int, []),
    "sg_decoder_variant_count": (C.c_int, []),
    "sg_decoder_variant_name": (C.c_char_p, [C.c_int]),
    "sg_decoder_set_variant": (C.c_int, [C.c_int]),
    "sg_decoder_get_variant": (C.c_int, []),
    "sg_status_string": (C.c_char_p, [C.c_int]),
    "sg_last_error": (C.c_char_p, []),
    "sg_version": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `make -C sogrand_b200/csrc` "
                "(there is no CPU fallback)"
            )
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def symbols() -> list[str]:
    return list(_SIGS)


class SograndError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def check(status: int) -> None:
    if status != 0:
        raise SograndError(status, load().sg_last_error().decode())

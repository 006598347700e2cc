"""ctypes binding of ``include/lfts_b200.h`` (``liblfts_b200.so``).

This is the Python face of the C ABI: every call goes into the CUDA library.
There is no CPU fallback -- if the library is missing or no GPU is visible,
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liblfts_b200.so")

LFTS_FP64 = 0
LFTS_FP32_MIXED = 1

# lfts_status codes that callers act on
LFTS_OK = 0
LFTS_ERR_SINGULAR = 5
LFTS_ERR_NOTCONV = 7
LFTS_ERR_NONFINITE = 8


class LftsError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        lib = _lib
        msg = lib.lfts_status_string(status).decode() if lib else str(status)
        extra = lib.lfts_last_error_string().decode() if lib else ""
        super().__init__(f"{what}: {msg}" + (f" ({extra})" if extra else ""))


class Params(C.Structure):
    _fields_ = [("N", C.c_int), ("NA", C.c_int), ("XbN", C.c_double), ("C", C.c_double),
                ("dt", C.c_double), ("m", C.c_int * 3), ("L", C.c_double * 3)]


class Input(C.Structure):
    _fields_ = [("N", C.c_int), ("NA", C.c_int), ("NB", C.c_int), ("XN_in", C.c_double),
                ("C", C.c_double), ("dt", C.c_double), ("isXeN", C.c_int), ("m", C.c_int * 3),
                ("L", C.c_double * 3), ("equil_its", C.c_int), ("sim_its", C.c_int),
                ("sample_freq", C.c_int), ("save_freq", C.c_int), ("loadType", C.c_int),
                ("XbN", C.c_double), ("XeN", C.c_double), ("V", C.c_double), ("sigma", C.c_double),
                ("M", C.c_longlong), ("Mk", C.c_longlong)]


class Tiles(C.Structure):
    _fields_ = [("pencil_cw", C.c_int), ("plane_stages", C.c_int), ("h_in_pencil", C.c_int),
                ("two_streams", C.c_int), ("phi_in_chain", C.c_int), ("plane_split", C.c_int)]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_P = C.c_void_p

# name -> (restype, argtypes); the full list of entry points include/lfts_b200.h declares
SIGNATURES = {
    "lfts_version": (C.c_char_p, []),
    "lfts_status_string": (C.c_char_p, [C.c_int]),
    "lfts_last_error_string": (C.c_char_p, []),
    "lfts_mesh_supported": (C.c_int, [C.c_int]),
    "lfts_create": (C.c_int, [C.POINTER(Params), C.c_int, C.c_int, C.POINTER(_P)]),
    "lfts_destroy": (C.c_int, [_P]),
    "lfts_device_bytes": (C.c_int, [_P, C.POINTER(C.c_size_t)]),
    "lfts_set_fields": (C.c_int, [_P, _dp]),
    "lfts_get_fields": (C.c_int, [_P, _dp]),
    "lfts_fields_device": (C.c_int, [_P, C.POINTER(C.c_void_p)]),
    "lfts_calc_concs": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "lfts_anderson_mix": (C.c_int, [_P, C.c_int, C.c_double, C.POINTER(C.c_int)]),
    "lfts_langevin_init": (C.c_int, [_P, _dp]),
    "lfts_langevin_step": (C.c_int, [_P, _dp]),
    "lfts_langevin_step_device": (C.c_int, [_P, C.c_void_p]),
    "lfts_langevin_full_step": (C.c_int, [_P, C.c_void_p, C.c_int, C.c_double, C.POINTER(C.c_int),
                                          C.POINTER(C.c_double)]),
    "lfts_sk_sample": (C.c_int, [_P]),
    "lfts_sk_get": (C.c_int, [_P, _dp, C.POINTER(C.c_int)]),
    "lfts_sk_reset": (C.c_int, [_P]),
    "lfts_sk_bin": (C.c_int, [_P, C.c_double, _dp, _dp, C.POINTER(C.c_int)]),
    "lfts_get_H": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "lfts_step_fwd": (C.c_int, [_P, _dp, _dp, _dp, C.c_int]),
    "lfts_g_lookup": (C.c_int, [_P, _dp]),
    "lfts_step_fwd_noalloc": (C.c_int, [C.POINTER(Params), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.c_void_p]),
    "lfts_backward": (C.c_int, [_P, C.c_int, _dp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "lfts_stream": (C.c_void_p, [_P]),
    "lfts_kernel_launches": (C.c_longlong, [_P]),
    "lfts_tuning": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "lfts_get_tiles": (C.c_int, [_P, C.POINTER(Tiles)]),
    "lfts_set_tiles": (C.c_int, [_P, C.POINTER(Tiles)]),
    "lfts_ensemble_tiles": (C.c_int, [_P, C.c_int, C.POINTER(Tiles)]),
    "lfts_profile_chain": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "lfts_profile_iteration": (C.c_int, [_P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double)]),
    "lfts_anderson_stats": (C.c_int, [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "lfts_get_propagators": (C.c_int, [_P, _dp]),
    "lfts_ensemble_create": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong), C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "lfts_ensemble_destroy": (C.c_int, [_P]),
    "lfts_ensemble_set_fields": (C.c_int, [_P, C.c_int, _dp]),
    "lfts_ensemble_get_fields": (C.c_int, [_P, C.c_int, _dp]),
    "lfts_ensemble_mix": (C.c_int, [_P, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "lfts_ensemble_run": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "lfts_ensemble_replica_status": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "lfts_ensemble_tuning": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int)]),
    "lfts_ensemble_stream": (C.c_void_p, [_P]),
    "lfts_ensemble_kernel_launches": (C.c_longlong, [_P]),
    "lfts_noise_philox": (C.c_int, [C.c_ulonglong, C.c_longlong, C.c_longlong, C.c_double, _dp]),
    "lfts_read_input": (C.c_int, [C.c_char_p, C.POINTER(Input)]),
    "lfts_z_inf_discrete": (C.c_double, [C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.c_double,
                                         C.c_int]),
    "lfts_params_from_input": (None, [C.POINTER(Input), C.POINTER(Params)]),
    "lfts_rng_create": (C.c_int, [C.c_ulonglong, C.c_double, C.POINTER(_P)]),
    "lfts_rng_destroy": (C.c_int, [_P]),
    "lfts_rng_normal": (C.c_int, [_P, C.c_longlong, _dp]),
    "lfts_rng_uniform": (C.c_int, [_P, C.c_longlong, _dp]),
    "lfts_lamellar_field": (C.c_int, [_dp, C.c_double, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int]),
    "lfts_random_field": (C.c_int, [_P, _dp, C.c_double, C.c_longlong]),
}


def lib():
    """Load liblfts_b200.so (building it first if it is absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        h = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def check(status: int, what: str) -> None:
    if status != 0:
        raise LftsError(status, what)


def check_mix(status: int, what: str, strict: bool) -> int:
    """As check(), except that an Anderson mix stopped at its iteration cap
    (LFTS_ERR_NOTCONV) is returned rather than raised unless ``strict``: the
    reference carries on past the cap, and so do callers that mirror it."""
    if status == LFTS_ERR_NOTCONV and not strict:
        return status
    check(status, what)
    return status

"""Loader for libqnd_b200.so (the CUDA engine behind include/qnd.h).

The library is built in-tree by ``tdse_nd_mpi_b200.build``. There is no CPU
fallback: if the library is missing this module raises, so a GPU run can never
silently route through something else.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libqnd_b200.so")

QND_OK, QND_EINVAL, QND_ECUDA, QND_ENOMEM, QND_ENORM, QND_EUNSUPPORTED, QND_ENONFINITE = 0, 1, 2, 3, 4, 5, 6
QND_FP64, QND_MIXED = 0, 1

# (name, argtypes) for every symbol declared in include/qnd.h
_vp, _ip, _dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
_i64, _i64p = C.c_int64, C.POINTER(C.c_int64)
_names = C.POINTER(C.c_char_p)
SIGNATURES = {
    "qnd_version": ([], C.c_char_p),
    "qnd_last_error": ([], C.c_char_p),
    "qnd_ctx_create": ([C.c_int, _i64p, _dp, C.c_char_p, C.c_double, C.c_int, C.POINTER(_vp)], C.c_int),
    "qnd_ctx_destroy": ([_vp], C.c_int),
    "qnd_ctx_set_stream": ([_vp, _vp], C.c_int),
    "qnd_ctx_info": ([_vp, _i64p, _ip, _dp, _dp, _dp], C.c_int),
    "qnd_state_bytes": ([_vp, _i64p], C.c_int),
    "qnd_set_potential_named": ([_vp, C.c_char_p], C.c_int),
    "qnd_set_potential": ([_vp, _dp], C.c_int),
    "qnd_set_cap": ([_vp, C.c_double, C.c_double], C.c_int),
    "qnd_set_vcap": ([_vp, _dp], C.c_int),
    "qnd_set_gradv": ([_vp, C.c_int, _dp], C.c_int),
    "qnd_set_mask_axis": ([_vp, C.c_int, _dp], C.c_int),
    "qnd_state_alloc": ([_vp, _i64, C.POINTER(_vp)], C.c_int),
    "qnd_state_free": ([_vp, _vp], C.c_int),
    "qnd_state_upload": ([_vp, _vp, _dp], C.c_int),
    "qnd_state_download": ([_vp, _dp, _vp], C.c_int),
    "qnd_synchronize": ([_vp], C.c_int),
    "qnd_step_imag": ([_vp, _vp, _i64], C.c_int),
    "qnd_step_length": ([_vp, _vp, _dp, _i64], C.c_int),
    "qnd_step_velocity": ([_vp, _vp, _dp, _i64], C.c_int),
    "qnd_to_p": ([_vp, _vp], C.c_int),
    "qnd_to_r": ([_vp, _vp], C.c_int),
    "qnd_run_length": ([_vp, _vp, _dp, _i64, C.c_int, _names, _dp], C.c_int),
    "qnd_run_velocity": ([_vp, _vp, _dp, _dp, _i64, C.c_int, _names, _dp], C.c_int),
    "qnd_gram_schmidt": ([_vp, C.POINTER(_vp), C.c_int, _dp], C.c_int),
    "qnd_imag_propagate": ([_vp, C.POINTER(_vp), C.c_int, _i64], C.c_int),
    "qnd_run_length_dev": ([_vp, _vp, _vp, _i64, C.c_int, _names, _vp], C.c_int),
    "qnd_ctx_set_profiling": ([_vp, C.c_int], C.c_int),
    "qnd_ctx_get_profile": ([_vp, _i64p, _i64p, _dp, C.c_int], C.c_int),
    "qnd_observable_count": ([_vp, C.c_int, _names, _ip], C.c_int),
    "qnd_observables": ([_vp, _vp, C.c_int, _names, _dp, _dp], C.c_int),
    "qnd_energies": ([_vp, _vp, C.c_int, _dp], C.c_int),
    "qnd_observables_rspace_noalloc": ([_vp, _vp, C.c_int, _names, _vp], C.c_int),
    "qnd_final_spectra": ([_vp, _vp, C.c_double, C.c_double, _dp, C.c_double, C.c_int, _dp, _i64p, _dp], C.c_int),
    "qnd_run_length_batch": ([C.c_int, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), _i64, C.c_int, _names,
                              C.POINTER(_vp)], C.c_int),
    "qnd_run_length_sweep": ([C.c_int, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), _i64, C.c_int, _names,
                              C.POINTER(_vp)], C.c_int),
    "qnd_adjoint_length": ([_vp, _vp, _dp, _i64, _dp, _i64, _dp, _dp, _vp], C.c_int),
    "qnd_adjoint_velocity": ([_vp, _vp, _dp, _i64, _dp, _i64, _dp, _dp, _vp], C.c_int),
    "qnd_field_samples": ([_vp, C.c_int, _vp, _i64, _vp, _vp, _vp, C.c_int], C.c_int),
    "qnd_state_embed": ([_vp, _vp, _dp, _i64p, C.c_double, C.c_double, C.c_int], C.c_int),
}

QND_ENV = {"constant": 0, "trapz": 1, "cos2": 2, "cos4": 3}


class LaserMode(C.Structure):
    """qnd_laser_mode: one mode as the reference holds it after parameters.c:805-810."""

    _fields_ = [("frequency", C.c_double), ("amplitude", C.c_double), ("ellipticity", C.c_double),
                ("cep", C.c_double), ("delay", C.c_double), ("duration", C.c_double), ("envelope", C.c_int)]

_lib = None


class QndError(RuntimeError):
    """A non-zero status from the C ABI (the reference would MPI_Abort)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[qnd error {code}] {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA engine first (python -m tdse_nd_mpi_b200.build); "
                "there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != QND_OK:
        raise QndError(rc, lib().qnd_last_error().decode(errors="replace"))

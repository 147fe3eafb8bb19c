"""ctypes binding of the engine's C ABI (include/fcib.h).

This is the binding a host program would add to call the engine; it loads the in-tree
libfcib200.so and raises when the library or a CUDA device is missing (there is no CPU
fallback).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfcib200.so")
_LIB = None

FCIB_OK = 0
FCIB_ERR_ARG = -1
FCIB_ERR_STATE = -2
FCIB_ERR_CUDA = -3
FCIB_ERR_UNSUPPORTED = -4
FCIB_ERR_NOT_CONVERGED = -5
FCIB_ERR_NUMERIC = -6

PREC_FP64 = 0
PREC_MIXED = 1
PREC_MIXED_TF32 = 2
PRECOND_DIAG = 0
PRECOND_MLP = 1
SAME_TC = 0
SAME_CUDA_CORES = 1


class FcibOptions(C.Structure):
    _fields_ = [
        ("maxiter", C.c_int),
        ("e_convergence", C.c_double),
        ("r_convergence", C.c_double),
        ("guess_per_root", C.c_int),
        ("dets_per_guess", C.c_int),
        ("collapse_per_root", C.c_int),
        ("subspace_per_root", C.c_int),
        ("die_if_not_converged", C.c_int),
        ("print_", C.c_int),
        ("precision", C.c_int),
        ("preconditioner", C.c_int),
        ("mixed_switch", C.c_double),
        ("same_spin_kernel", C.c_int),
        ("spin_adapt", C.c_int),
        ("sym_blocked", C.c_int),
        ("spin_adapt_full_preconditioner", C.c_int),
    ]


class FcibProfile(C.Structure):
    _fields_ = [
        ("total_ms", C.c_double), ("sigma_ms", C.c_double), ("ab_ms", C.c_double), ("same_ms", C.c_double),
        ("ab64_ms", C.c_double), ("same64_ms", C.c_double),
        ("guess_ms", C.c_double), ("iterations", C.c_int), ("n_sigma", C.c_int), ("n_sigma_fp64", C.c_int),
        ("n_ab", C.c_int), ("n_ab64", C.c_int), ("launches", C.c_ulonglong), ("tc_kernel_ms", C.c_double),
    ]


class FcibError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fcib error {code}: {msg}")
        self.code = code


#: exported symbols and their (restype, argtypes)
_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_up = C.POINTER(C.c_uint32)
_vp = C.c_void_p
SIGNATURES = {
    "fcib_default_options": (None, [C.POINTER(FcibOptions)]),
    "fcib_last_error": (C.c_char_p, []),
    "fcib_version": (C.c_char_p, []),
    "fcib_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "fcib_destroy": (C.c_int, [_vp]),
    "fcib_set_integrals": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_double, _dp, _dp, _dp, _dp, _dp]),
    "fcib_set_state": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
    "fcib_set_options": (C.c_int, [_vp, C.POINTER(FcibOptions)]),
    "fcib_size": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "fcib_layout_size": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "fcib_set_gas": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fcib_determinants": (C.c_int, [_vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "fcib_ncsf": (C.c_int, [_vp, C.POINTER(C.c_int64)]),
    "fcib_csf_to_det": (C.c_int, [_vp, _dp, _dp]),
    "fcib_det_to_csf": (C.c_int, [_vp, _dp, _dp]),
    "fcib_csf_hdiag": (C.c_int, [_vp, C.c_int, _dp]),
    "fcib_solve": (C.c_int, [_vp, _dp, _dp, C.POINTER(C.c_int)]),
    "fcib_reset_guess": (C.c_int, [_vp]),
    "fcib_get_vector": (C.c_int, [_vp, C.c_int, _dp]),
    "fcib_sigma": (C.c_int, [_vp, _dp, _dp]),
    "fcib_sigma_device": (C.c_int, [_vp, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]),
    "fcib_hdiag": (C.c_int, [_vp, _dp]),
    "fcib_spin2": (C.c_int, [_vp, _dp, _dp]),
    "fcib_rdms": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    "fcib_compute_rdms": (C.c_int, [_vp, _dp, _dp, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp]),
    "fcib_rdms3": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp]),
    "fcib_csf_coupling": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, _dp, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fcib_compute_rdms3": (C.c_int, [_vp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp]),
    "fcib_num_strings": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_int64)]),
    "fcib_strings": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_uint32)]),
    "fcib_string_list": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int8), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]),
    "fcib_last_timing": (C.c_int, [_vp, _dp, C.POINTER(C.c_int), _dp]),
    "fcib_get_profile": (C.c_int, [_vp, C.POINTER(FcibProfile)]),
    "fcib_stream": (C.c_int, [_vp, C.POINTER(C.c_void_p)]),
    "fcib_spin2_device_noalloc": (C.c_int, [_vp, C.c_void_p, _dp, C.c_void_p]),
    "fcib_set_mlp": (C.c_int, [_vp, _fp, C.c_int]),
    "fcib_mlp_eval": (C.c_int, [C.c_int, C.c_int64, _up, _up, _fp, _fp, _fp, _fp]),
    "fcib_mlp_grad": (C.c_int, [C.c_int, C.c_int64, _up, _up, _fp, _fp, _fp, _fp, _fp, _fp, _dp]),
    "fcib_mlp_train": (C.c_int, [C.c_int, C.c_int64, _up, _up, _fp, _fp, _fp, _fp, C.c_int, C.c_int, C.c_float,
                                 C.c_uint64, C.c_int, _fp, _dp]),
    "fcib_precondition": (C.c_int, [_vp, _dp, C.c_double, _dp]),
    "fcib_set_residual_capture": (C.c_int, [_vp, C.c_int]),
    "fcib_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int), _dp, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp),
                                    C.POINTER(_dp), C.POINTER(_dp), C.c_int, C.POINTER(FcibOptions)]),
    "fcib_batch_destroy": (C.c_int, [_vp]),
    "fcib_batch_solve": (C.c_int, [_vp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]),
    "fcib_batch_set_shape": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "fcib_batch_phase_cycles": (C.c_int, [C.POINTER(C.c_ulonglong)]),
    "fcib_batch_tune": (C.c_int, [_vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), _dp]),
    "fcib_captured_residual": (C.c_int, [_vp, C.c_int, _dp, _dp, C.POINTER(C.c_int)]),
    "fcib_fp64_peak": (C.c_int, [C.c_int, _dp, _dp]),
    "fcib_transition_rdms": (C.c_int, [_vp, C.c_int, _vp, C.c_int, C.c_int, C.c_int, _dp, _dp]),
    "fcib_max_abs_elements": (C.c_int, [_vp, C.c_int, C.c_int, _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
}
MLP_NWEIGHTS = 10689


def lib():
    """Loads libfcib200.so (built in-tree by forte_b200.build)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FcibError(FCIB_ERR_STATE, f"{LIB_PATH} is missing: run forte_b200.build.build() first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(rc):
    if rc != FCIB_OK:
        raise FcibError(rc, lib().fcib_last_error().decode())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(_fp)


def uptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_up)


def default_options() -> FcibOptions:
    o = FcibOptions()
    lib().fcib_default_options(C.byref(o))
    return o

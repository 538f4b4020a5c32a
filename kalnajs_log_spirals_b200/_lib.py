"""ctypes binding of libkls.so (include/kls.h).

The shared library is built in-tree (``kalnajs_log_spirals_b200/libkls.so``).
There is no CPU fallback: if the library is missing or has no CUDA device to
run on, the calls raise ``KlsError``.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkls.so")
# the same sources built with KLS_CHECKED (guarded accesses, kls_bounds_report)
CHECKED_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkls_checked.so")

KLS_OK = 0
KLS_ERR_CONFIG = 1
KLS_ERR_CUDA = 2
KLS_ERR_OOM = 3
KLS_ERR_STATE = 4
KLS_ERR_NONFINITE = 5
KLS_ERR_SINGULAR = 6
KLS_ERR_UNSUPPORTED = 7
KLS_ERR_TIMEOUT = 8

KLS_MODE_FP64 = 0
KLS_MODE_MIXED = 1
KLS_MODE_ANCHORED = 2
KLS_F64_4M = 0
KLS_F64_3M = 1

KLS_QUAD_DEFAULT = 0
KLS_QUAD_TRAPEZOID = 1
KLS_QUAD_SIMPSON = 2
KLS_QUAD_BOOLE = 3
QUAD_CODES = {"t": KLS_QUAD_TRAPEZOID, "s": KLS_QUAD_SIMPSON, "b": KLS_QUAD_BOOLE}

KLS_MIXED_AUTO = 0
KLS_MIXED_ONE_CTA = 1
KLS_MIXED_PAIR = 2
KLS_MIXED_TMEM = 3

KLS_FAULT_NONE = 0
KLS_FAULT_SKIP_ARRIVAL = 1
KLS_FAULT_NAN_ROW = 2

KLS_LU_AUTO = 0
KLS_LU_CTA = 1
KLS_LU_CLUSTER = 2

STATUS_NAMES = {0: "KLS_OK", 1: "KLS_ERR_CONFIG", 2: "KLS_ERR_CUDA", 3: "KLS_ERR_OOM",
                4: "KLS_ERR_STATE", 5: "KLS_ERR_NONFINITE", 6: "KLS_ERR_SINGULAR",
                7: "KLS_ERR_UNSUPPORTED", 8: "KLS_ERR_TIMEOUT"}


class KlsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class kls_config(C.Structure):
    _fields_ = [("m", C.c_int32), ("G", C.c_double), ("L0", C.c_double), ("n_zang", C.c_int32),
                ("q1", C.c_double), ("NR", C.c_int32), ("Ne", C.c_int32),
                ("Rc_min", C.c_double), ("Rc_max", C.c_double), ("v_min", C.c_double),
                ("N_alpha", C.c_int32), ("alpha_max", C.c_double), ("l_min", C.c_int32),
                ("l_max", C.c_int32), ("nw", C.c_int32), ("nwa", C.c_int32),
                ("quad_alpha", C.c_int32), ("quad_rc", C.c_int32), ("quad_v", C.c_int32)]


class kls_dims(C.Structure):
    _fields_ = [("NPh", C.c_int32), ("n_l", C.c_int32), ("N_alpha", C.c_int32),
                ("N_alpha_pad", C.c_int32), ("K", C.c_int64), ("K_pad", C.c_int64),
                ("nwa", C.c_int32), ("device_bytes", C.c_int64)]


class kls_newton_cfg(C.Structure):
    _fields_ = [("max_iter", C.c_int32), ("tol", C.c_double), ("delta", C.c_double),
                ("use_line_search", C.c_int32), ("max_line_search", C.c_int32),
                ("mode", C.c_int32)]


class kls_newton_result(C.Structure):
    _fields_ = [("Omega_p", C.c_double), ("gamma", C.c_double), ("omega_re", C.c_double),
                ("omega_im", C.c_double), ("det_re", C.c_double), ("det_im", C.c_double),
                ("iterations", C.c_int32), ("converged", C.c_int32), ("det_evals", C.c_int32)]


class kls_hybrid_cfg(C.Structure):
    _fields_ = [("mixed_delta", C.c_double), ("mixed_step_tol", C.c_double),
                ("mixed_max_iter", C.c_int32), ("fp64_max_iter", C.c_int32),
                ("anchor_radius", C.c_double), ("final_fp64", C.c_int32),
                ("far_step", C.c_double)]


class kls_scan_cfg(C.Structure):
    _fields_ = [("n_Op", C.c_int32), ("n_gamma", C.c_int32), ("Omega_p_min", C.c_double),
                ("Omega_p_max", C.c_double), ("gamma_min", C.c_double),
                ("gamma_max", C.c_double), ("mode", C.c_int32), ("batch", C.c_int32)]


class kls_multi_info(C.Structure):
    _fields_ = [("n_models", C.c_int32), ("batch", C.c_int32), ("mode", C.c_int32),
                ("n_items", C.c_int32), ("grid", C.c_int32), ("graph", C.c_int32),
                ("launches_per_replay", C.c_int32), ("replays", C.c_int64),
                ("last_ms", C.c_double), ("schedule", C.c_int32),
                ("schedule_ms", C.c_double * 2)]


class kls_tune_result(C.Structure):
    _fields_ = [("mode", C.c_int32), ("splits", C.c_int32), ("default_splits", C.c_int32),
                ("candidates", C.c_int32), ("ms_per_omega", C.c_double),
                ("default_ms_per_omega", C.c_double), ("form", C.c_int32)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)

# name -> (restype, argtypes); every symbol include/kls.h declares
SIGNATURES = {
    "kls_create": (C.c_int, [C.POINTER(kls_config), C.c_int, C.POINTER(_P)]),
    "kls_destroy": (C.c_int, [_P]),
    "kls_last_error": (C.c_char_p, [_P]),
    "kls_create_error": (C.c_char_p, []),
    "kls_get_dims": (C.c_int, [_P, C.POINTER(kls_dims)]),
    "kls_set_stream": (C.c_int, [_P, _P]),
    "kls_precompute": (C.c_int, [_P]),
    "kls_prepare_mixed": (C.c_int, [_P]),
    "kls_release_fp64": (C.c_int, [_P]),
    "kls_export_orbits": (C.c_int, [_P] + [_D] * 10),
    "kls_export_grids": (C.c_int, [_P] + [_D] * 6),
    "kls_export_alpha": (C.c_int, [_P] + [_D] * 3),
    "kls_export_resonant": (C.c_int, [_P] + [_D] * 2),
    "kls_export_W": (C.c_int, [_P, C.c_int, C.c_int, _D]),
    "kls_det_batch": (C.c_int, [_P, _D, C.c_int, C.c_int, _D, _D]),
    "kls_det_batch_device": (C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P]),
    "kls_build_M": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _D]),
    "kls_set_anchor": (C.c_int, [_P, C.c_double, C.c_double, _D]),
    "kls_det": (C.c_int, [_P, C.c_double, C.c_double, C.c_int, _D, _D, _D]),
    "kls_set_f64_form": (C.c_int, [_P, C.c_int]),
    "kls_scan": (C.c_int, [_P, C.POINTER(kls_scan_cfg), _D, _D, _D, _D]),
    "kls_newton": (C.c_int, [_P, C.c_double, C.c_double, C.POINTER(kls_newton_cfg),
                             C.POINTER(kls_newton_result), _D]),
    "kls_newton_hybrid": (C.c_int, [_P, C.c_double, C.c_double, C.POINTER(kls_newton_cfg),
                                    C.POINTER(kls_hybrid_cfg), C.POINTER(kls_newton_result),
                                    C.POINTER(C.c_int32), _D]),
    "kls_det_lu_static": (C.c_int, [_P, C.c_int, C.c_int, _P, _P, _P]),
    "kls_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(_P)]),
    "kls_mlp_destroy": (C.c_int, [_P]),
    "kls_mlp_num_params": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "kls_mlp_get_params": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "kls_mlp_set_params": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "kls_mlp_forward": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int, C.POINTER(C.c_float)]),
    "kls_mlp_grad": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                               C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "kls_mlp_train": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int,
                                C.c_int, C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "kls_multi_create": (C.c_int, [C.POINTER(_P), C.c_int, C.c_int, C.c_int, C.POINTER(_P)]),
    "kls_multi_destroy": (C.c_int, [_P]),
    "kls_multi_last_error": (C.c_char_p, [_P]),
    "kls_multi_det": (C.c_int, [_P, _D, C.c_int, _D, _D]),
    "kls_scan_multi": (C.c_int, [_P, C.POINTER(kls_scan_cfg), _D, _D, _D, _D]),
    "kls_multi_get_info": (C.c_int, [_P, C.POINTER(kls_multi_info)]),
    "kls_autotune": (C.c_int, [_P, C.c_int, C.c_int, C.POINTER(kls_tune_result)]),
    "kls_set_splits": (C.c_int, [_P, C.c_int, C.c_int]),
    "kls_set_lu_mode": (C.c_int, [_P, C.c_int]),
    "kls_set_mixed_form": (C.c_int, [_P, C.c_int]),
    "kls_set_mixed_chunk": (C.c_int, [_P, C.c_int]),
    "kls_set_wait_limit": (C.c_int, [_P, C.c_double]),
    "kls_set_fault_injection": (C.c_int, [_P, C.c_int]),
    "kls_enable_timing": (C.c_int, [_P, C.c_int]),
    "kls_get_stage_ms": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "kls_get_precompute_ms": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "kls_launch_count": (C.c_int64, [_P]),
    "kls_bounds_report": (C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.c_int]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libkls.so once; raises KlsError if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    _lib = _bind(path)
    return _lib


def load_checked(path: str = CHECKED_LIB_PATH) -> C.CDLL:
    """The bounds-checked build (a separate library object, not cached as
    the default); raises KlsError if it is missing."""
    return _bind(path)


def _bind(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise KlsError(KLS_ERR_STATE, f"{path} is missing: build it with "
                                      "`python -m kalnajs_log_spirals_b200.build`")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def dptr(a) -> _D:
    """double* of a contiguous (C or Fortran order) float64 or complex128 numpy
    array, or NULL for None; anything else raises TypeError (the library
    would read or write it as doubles)."""
    if a is None:
        return C.cast(None, _D)
    if a.dtype.name not in ("float64", "complex128") or not (a.flags.c_contiguous
                                                           or a.flags.f_contiguous):
        raise TypeError(f"expected a contiguous float64/complex128 array, got {a.dtype} "
                        f"(C {a.flags.c_contiguous}, F {a.flags.f_contiguous})")
    return a.ctypes.data_as(_D)


def check(ctx, code: int) -> None:
    if code != KLS_OK:
        lib = load()
        msg = lib.kls_last_error(ctx).decode() if ctx else lib.kls_create_error().decode()
        raise KlsError(code, msg)

"""ctypes bindings of libcyclops_b200.so (include/cyclops_b200.h).

The library is loaded from cyclops_b200/_lib/.  A missing library is an
error: there is no CPU fallback behind these functions.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcyclops_b200.so")

CYC_OK = 0
STATUS_NAMES = {1: "ARGUMENT", 2: "CUDA", 3: "MEMORY", 4: "UNSUPPORTED", 5: "STATE", 6: "TIMEOUT"}


class CyclopsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{STATUS_NAMES.get(status, status)}] {msg}")
        self.status = status


class DataDesc(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("K", C.c_int), ("J", C.c_int),
        ("pid", C.c_void_p), ("y", C.c_void_p), ("time", C.c_void_p),
        ("col_format", C.c_void_p), ("col_ptr", C.c_void_p), ("col_idx", C.c_void_p),
        ("val_ptr", C.c_void_p), ("col_val", C.c_void_p),
        ("has_offset", C.c_int), ("has_intercept", C.c_int),
    ]


class Control(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double), ("max_iterations", C.c_int), ("convergence_type", C.c_int),
        ("initial_bound", C.c_double), ("max_bound_count", C.c_int), ("precision", C.c_int),
        ("polish_tolerance", C.c_double), ("use_kkt_swindle", C.c_int),
    ]


class Prior(C.Structure):
    _fields_ = [("prior_type", C.c_int), ("exclude", C.c_void_p), ("n_exclude", C.c_int)]


class FitSpec(C.Structure):
    _fields_ = [("weights", C.c_void_p), ("variance", C.c_double), ("start_beta", C.c_void_p),
                ("fixed", C.c_void_p), ("n_fixed", C.c_int)]


class FitResult(C.Structure):
    _fields_ = [("beta", C.c_void_p), ("log_likelihood", C.c_double), ("log_prior", C.c_double),
                ("iterations", C.c_int), ("return_flag", C.c_int)]


class RunStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_double), ("algorithmic_bytes", C.c_double),
                ("gradient_entries", C.c_double), ("update_entries", C.c_double),
                ("coordinate_steps", C.c_double), ("index_entries", C.c_double), ("cycles", C.c_double),
                ("launches", C.c_int), ("phases", C.c_int), ("phase_ms", C.c_double * 2),
                ("phase_bytes", C.c_double * 2), ("phase_state_bytes", C.c_int * 2),
                ("cluster_ctas", C.c_int), ("batch_cap", C.c_int), ("batch_shared_rows", C.c_int),
                ("batch_levels", C.c_int)]


# name -> argtypes (all return int status unless listed in _RESTYPE)
_SIGS = {
    "cyc_last_error": [],
    "cyc_version": [],
    "cyc_dataset_create": [C.POINTER(DataDesc), C.c_int, C.POINTER(C.c_void_p)],
    "cyc_dataset_destroy": [C.c_void_p],
    "cyc_dataset_info": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                         C.POINTER(C.c_size_t)],
    "cyc_engine_create": [C.c_void_p, C.POINTER(C.c_void_p)],
    "cyc_engine_destroy": [C.c_void_p],
    "cyc_engine_clone": [C.c_void_p, C.POINTER(C.c_void_p)],
    "cyc_engine_set_weights": [C.c_void_p, C.c_void_p, C.c_int],
    "cyc_engine_compute_fixed_terms_ll": [C.c_void_p, C.c_int],
    "cyc_engine_compute_fixed_terms_gh": [C.c_void_p, C.c_int],
    "cyc_engine_zero_xbeta": [C.c_void_p],
    "cyc_engine_axpy_xbeta": [C.c_void_p, C.c_double, C.c_int],
    "cyc_engine_compute_xbeta": [C.c_void_p, C.c_void_p, C.c_int],
    "cyc_engine_compute_remaining_statistics": [C.c_void_p, C.c_int],
    "cyc_engine_compute_numerator_for_gradient": [C.c_void_p, C.c_int, C.c_int],
    "cyc_engine_compute_gradient_and_hessian": [C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                                C.POINTER(C.c_double), C.c_int],
    "cyc_engine_update_xbeta": [C.c_void_p, C.c_double, C.c_int, C.c_int],
    "cyc_engine_get_log_likelihood": [C.c_void_p, C.c_int, C.POINTER(C.c_double)],
    "cyc_engine_get_gradient_objective": [C.c_void_p, C.c_int, C.POINTER(C.c_double)],
    "cyc_engine_get_predictive_log_likelihood": [C.c_void_p, C.c_void_p, C.POINTER(C.c_double)],
    "cyc_engine_get_predictive_estimates": [C.c_void_p, C.c_void_p, C.c_void_p],
    "cyc_engine_get_xbeta": [C.c_void_p, C.c_void_p],
    "cyc_engine_save_xbeta": [C.c_void_p],
    "cyc_engine_get_xbeta_save": [C.c_void_p, C.c_void_p],
    "cyc_engine_get_n": [C.c_void_p, C.POINTER(C.c_int)],
    "cyc_engine_fisher_information": [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "cyc_fit": [C.c_void_p, C.POINTER(Prior), C.POINTER(FitSpec), C.POINTER(Control), C.POINTER(FitResult)],
    "cyc_batch_fit": [C.c_void_p, C.POINTER(Prior), C.POINTER(FitSpec), C.c_int, C.POINTER(Control),
                      C.POINTER(FitResult)],
    "cyc_last_run_stats": [C.POINTER(RunStats)],
    "cyc_cv_fold_weights": [C.c_int, C.c_void_p, C.c_int, C.c_long, C.c_int, C.c_int, C.c_void_p],
    "cyc_bootstrap_weights": [C.c_int, C.c_void_p, C.c_int, C.c_long, C.c_void_p, C.c_void_p],
    "cyc_launch_count": [],
    "cyc_gradient_hessian_noalloc": [C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p],
    "cyc_cv_grid_fit": [C.c_void_p, C.POINTER(Prior), C.c_void_p, C.c_int, C.c_void_p, C.c_int,
                        C.POINTER(Control), C.POINTER(FitResult), C.c_void_p, C.c_void_p],
    "cyc_fit_host_loop": [C.c_void_p, C.POINTER(Prior), C.POINTER(FitSpec), C.POINTER(Control),
                          C.POINTER(FitResult)],
    "cyc_profile_log_likelihood": [C.c_void_p, C.POINTER(Prior), C.POINTER(FitSpec), C.POINTER(Control), C.c_int,
                                   C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "cyc_profile_log_likelihood_batch": [C.c_void_p, C.POINTER(Prior), C.POINTER(FitSpec), C.POINTER(Control),
                                         C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p],
    "cyc_cv_grid_fit_weighted": [C.c_void_p, C.POINTER(Prior), C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                 C.POINTER(Control), C.POINTER(FitResult), C.c_void_p, C.c_void_p],
    "cyc_cv_auto_search": [C.c_void_p, C.POINTER(Prior), C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_double,
                           C.POINTER(Control), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p, C.c_void_p,
                           C.c_void_p, C.c_int, C.POINTER(C.c_int)],
    "cyc_ingest_covariates": [C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                              C.POINTER(C.c_void_p)],
    "cyc_ingest_sizes": [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "cyc_ingest_copy": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "cyc_ingest_free": [C.c_void_p],
    "cyc_profile_bounds": [C.c_void_p, C.POINTER(Prior), C.POINTER(FitSpec), C.POINTER(Control), C.c_void_p,
                           C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.POINTER(FitResult)],
}
_RESTYPE = {"cyc_last_error": C.c_char_p, "cyc_launch_count": C.c_longlong, "cyc_ingest_free": None}

_lock = threading.Lock()
_lib = None


def lib() -> C.CDLL:
    """The loaded library; raises if it has not been built."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `python -m cyclops_b200.build` "
                    "(there is no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, args in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = _RESTYPE.get(name, C.c_int)
            _lib = L
        return _lib


def exported_symbols():
    return list(_SIGS)


def check(status: int) -> None:
    if status != CYC_OK:
        raise CyclopsError(status, lib().cyc_last_error().decode(errors="replace"))

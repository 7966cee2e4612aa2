"""cyclops_b200: the Cyclops CCD inner loop on B200 (sm_100a).

The CUDA library (cyclops_b200/_lib/libcyclops_b200.so, C ABI in
include/cyclops_b200.h) holds all compute; this package is its host side:
the column store and synthetic generators (`data`), ctypes bindings
(`_native`) and an API mirroring the reference's user surface (`api`).
"""
from . import data  # noqa: F401
from .api import (Dataset, Engine, FitResult, batch_fit, create_control, create_prior,  # noqa: F401
                  cv_fold_weights, fit_cyclops_model, last_run_stats)

__all__ = ["data", "Dataset", "Engine", "FitResult", "batch_fit", "create_control", "create_prior",
           "cv_fold_weights", "fit_cyclops_model", "last_run_stats"]

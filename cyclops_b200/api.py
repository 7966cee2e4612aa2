"""Host API mirroring the reference's user-facing surface for this path.

    data    = cyclops_b200.data.CyclopsData(...)          # createCyclopsData
    prior   = create_prior("laplace", variance=200)       # createPrior (R/ModelFit.R:574)
    control = create_control(tolerance=1e-6)              # createControl (R/ModelFit.R:489)
    fit     = fit_cyclops_model(data, prior, control)     # fitCyclopsModel (R/ModelFit.R:65)

plus `Engine`, the per-coordinate AbstractModelSpecifics surface, and
`batch_fit`, many fits sharing one dataset on the GPU.  Every call goes
through libcyclops_b200.so; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import statistics
from typing import List, Optional, Sequence

import numpy as np

from . import _native as N
from .data import (CONV_GRADIENT, CONV_LANGE, CONV_MITTAL, CONV_ONE_STEP, CONV_ZHANG_OLES,
                   PRIOR_LAPLACE, PRIOR_NONE, PRIOR_NORMAL, CyclopsData)

FP64, MIXED = 0, 1

_PRIORS = {"none": PRIOR_NONE, "laplace": PRIOR_LAPLACE, "normal": PRIOR_NORMAL}
_CONV = {"gradient": CONV_GRADIENT, "lange": CONV_LANGE, "mittal": CONV_MITTAL,
         "onestep": CONV_ONE_STEP, "zhang-oles": CONV_ZHANG_OLES}


@dataclasses.dataclass
class PriorSpec:
    prior_type: int = PRIOR_LAPLACE
    variance: float = 1.0
    exclude: Optional[Sequence[int]] = None      # None: exclude the intercept
    force_intercept: bool = False


def create_prior(prior_type: str = "none", variance: float = 1.0, exclude=None,
                 force_intercept: bool = False) -> PriorSpec:
    """createPrior (R/ModelFit.R:574-617).  `variance` is the prior variance;
    a Laplace prior has rate lambda = sqrt(2/variance)."""
    if prior_type not in _PRIORS:
        raise ValueError(f"unknown prior type {prior_type!r}")
    return PriorSpec(_PRIORS[prior_type], float(variance), exclude, force_intercept)


@dataclasses.dataclass
class ControlSpec:
    tolerance: float = 1e-6
    max_iterations: int = 1000
    convergence_type: int = CONV_GRADIENT
    initial_bound: float = 2.0
    max_bound_count: int = 5
    precision: int = FP64
    polish_tolerance: float = 1e-4
    use_kkt_swindle: bool = False


def create_control(tolerance=1e-6, max_iterations=1000, convergence_type="gradient",
                   initial_bound=2.0, max_bound_count=5, precision="fp64",
                   polish_tolerance=1e-4, use_kkt_swindle=False) -> ControlSpec:
    """createControl (R/ModelFit.R:489-540); defaults are the reference's.
    `use_kkt_swindle` is createControl's useKKTSwindle: fit_cyclops_model
    then runs the reference's active-set passes under a Laplace prior."""
    ct = _CONV[convergence_type] if isinstance(convergence_type, str) else int(convergence_type)
    pr = {"fp64": FP64, "mixed": MIXED}[precision] if isinstance(precision, str) else int(precision)
    return ControlSpec(tolerance, max_iterations, ct, initial_bound, max_bound_count, pr,
                       polish_tolerance, bool(use_kkt_swindle))


def _exclude_for(data: CyclopsData, prior: PriorSpec) -> List[int]:
    """The intercept is excluded from regularisation unless forced
    (R/ModelFit.R:120-144)."""
    if prior.exclude is not None:
        return list(prior.exclude)
    if prior.prior_type != PRIOR_NONE and data.has_intercept and not prior.force_intercept:
        return [1 if data.has_offset else 0]
    return []


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


class Dataset:
    """A CyclopsData copied to device `device` (cyc_dataset_create)."""

    def __init__(self, data: CyclopsData, device: int = 0):
        self.data = data
        self.device = device
        keep = {
            "pid": None if data.pid is None else np.ascontiguousarray(data.pid, np.int32),
            "y": np.ascontiguousarray(data.y, np.float64),
            "time": None if data.time is None else np.ascontiguousarray(data.time, np.float64),
            "fmt": np.ascontiguousarray(data.col_format, np.int32),
            "cp": np.ascontiguousarray(data.col_ptr, np.int64),
            "ci": np.ascontiguousarray(data.col_idx, np.int32),
            "vp": np.ascontiguousarray(data.val_ptr, np.int64),
            "cv": np.ascontiguousarray(data.col_val, np.float64),
        }
        d = N.DataDesc(model=data.model, K=data.K, J=data.J, pid=_ptr(keep["pid"]), y=_ptr(keep["y"]),
                       time=_ptr(keep["time"]), col_format=_ptr(keep["fmt"]), col_ptr=_ptr(keep["cp"]),
                       col_idx=_ptr(keep["ci"]) if data.nnz else None, val_ptr=_ptr(keep["vp"]),
                       col_val=_ptr(keep["cv"]) if keep["cv"].size else None,
                       has_offset=int(data.has_offset), has_intercept=int(data.has_intercept))
        h = C.c_void_p()
        N.check(N.lib().cyc_dataset_create(C.byref(d), device, C.byref(h)))
        self.handle = h

    def info(self):
        K, J, nnz, b = C.c_int(), C.c_int(), C.c_longlong(), C.c_size_t()
        N.check(N.lib().cyc_dataset_info(self.handle, C.byref(K), C.byref(J), C.byref(nnz), C.byref(b)))
        return {"K": K.value, "J": J.value, "nnz": nnz.value, "device_bytes": b.value}

    def close(self):
        if getattr(self, "handle", None):
            N.lib().cyc_dataset_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Engine:
    """The AbstractModelSpecifics surface (src/cyclops/engine/AbstractModelSpecifics.h:46-122)."""

    def __init__(self, dataset: Dataset, _handle=None):
        self.dataset = dataset
        if _handle is None:
            h = C.c_void_p()
            N.check(N.lib().cyc_engine_create(dataset.handle, C.byref(h)))
            _handle = h
        self.handle = _handle
        self.K = dataset.data.K
        self.J = dataset.data.J

    def clone(self) -> "Engine":
        h = C.c_void_p()
        N.check(N.lib().cyc_engine_clone(self.handle, C.byref(h)))
        return Engine(self.dataset, h)

    def set_weights(self, w=None, use_cv=None):
        self._w = None if w is None else np.ascontiguousarray(w, np.float64)
        uc = int(w is not None) if use_cv is None else int(use_cv)
        N.check(N.lib().cyc_engine_set_weights(self.handle, _ptr(self._w), uc))

    def compute_fixed_terms_in_log_likelihood(self, use_cv=False):
        N.check(N.lib().cyc_engine_compute_fixed_terms_ll(self.handle, int(use_cv)))

    def compute_fixed_terms_in_gradient_and_hessian(self, use_cv=False):
        N.check(N.lib().cyc_engine_compute_fixed_terms_gh(self.handle, int(use_cv)))

    def zero_xbeta(self):
        N.check(N.lib().cyc_engine_zero_xbeta(self.handle))

    def axpy_xbeta(self, beta: float, j: int):
        N.check(N.lib().cyc_engine_axpy_xbeta(self.handle, float(beta), int(j)))

    def compute_xbeta(self, beta, use_w=False):
        b = np.ascontiguousarray(beta, np.float64)
        N.check(N.lib().cyc_engine_compute_xbeta(self.handle, _ptr(b), int(use_w)))

    def compute_remaining_statistics(self, use_w=False):
        N.check(N.lib().cyc_engine_compute_remaining_statistics(self.handle, int(use_w)))

    def compute_numerator_for_gradient(self, j, use_w=False):
        N.check(N.lib().cyc_engine_compute_numerator_for_gradient(self.handle, int(j), int(use_w)))

    def compute_gradient_and_hessian(self, j, use_w=False):
        g, h = C.c_double(), C.c_double()
        N.check(N.lib().cyc_engine_compute_gradient_and_hessian(self.handle, int(j), C.byref(g),
                                                                C.byref(h), int(use_w)))
        return g.value, h.value

    def update_xbeta(self, delta, j, use_w=False):
        N.check(N.lib().cyc_engine_update_xbeta(self.handle, float(delta), int(j), int(use_w)))

    def get_log_likelihood(self, use_cv=False):
        v = C.c_double()
        N.check(N.lib().cyc_engine_get_log_likelihood(self.handle, int(use_cv), C.byref(v)))
        return v.value

    def get_gradient_objective(self, use_cv=False):
        v = C.c_double()
        N.check(N.lib().cyc_engine_get_gradient_objective(self.handle, int(use_cv), C.byref(v)))
        return v.value

    def get_predictive_log_likelihood(self, w):
        w = np.ascontiguousarray(w, np.float64)
        v = C.c_double()
        N.check(N.lib().cyc_engine_get_predictive_log_likelihood(self.handle, _ptr(w), C.byref(v)))
        return v.value

    def get_predictive_estimates(self, w=None):
        y = np.zeros(self.K)
        ww = None if w is None else np.ascontiguousarray(w, np.float64)
        N.check(N.lib().cyc_engine_get_predictive_estimates(self.handle, _ptr(y), _ptr(ww)))
        return y

    def get_xbeta(self):
        out = np.zeros(self.K)
        N.check(N.lib().cyc_engine_get_xbeta(self.handle, _ptr(out)))
        return out

    def save_xbeta(self):
        N.check(N.lib().cyc_engine_save_xbeta(self.handle))

    def get_xbeta_save(self):
        out = np.zeros(self.K)
        N.check(N.lib().cyc_engine_get_xbeta_save(self.handle, _ptr(out)))
        return out

    def fisher_information(self, columns, use_cv=False) -> np.ndarray:
        """computeFisherInformation for every pair of `columns` at the current
        coefficients (CyclicCoordinateDescent.cpp:1288-1300): n x n."""
        cols = np.ascontiguousarray(columns, np.int32)
        out = np.zeros((cols.size, cols.size))
        N.check(N.lib().cyc_engine_fisher_information(self.handle, _ptr(cols), int(cols.size), int(use_cv),
                                                      _ptr(out)))
        return out

    def n_denominators(self) -> int:
        n = C.c_int()
        N.check(N.lib().cyc_engine_get_n(self.handle, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "handle", None):
            N.lib().cyc_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclasses.dataclass
class FitResult:
    beta: np.ndarray
    log_likelihood: float
    log_prior: float
    iterations: int
    return_flag: int


def _control_struct(c: ControlSpec) -> N.Control:
    return N.Control(tolerance=c.tolerance, max_iterations=c.max_iterations,
                     convergence_type=c.convergence_type, initial_bound=c.initial_bound,
                     max_bound_count=c.max_bound_count, precision=c.precision,
                     polish_tolerance=c.polish_tolerance, use_kkt_swindle=int(c.use_kkt_swindle))


def _prior_struct(data: CyclopsData, prior: PriorSpec):
    ex = np.ascontiguousarray(_exclude_for(data, prior), np.int32)
    return N.Prior(prior_type=prior.prior_type, exclude=_ptr(ex) if ex.size else None,
                   n_exclude=int(ex.size)), ex


def _fixed_columns(fixed, J: int) -> Optional[np.ndarray]:
    """fixedCoefficients as column ids: a boolean mask of length J or a list
    of ids (None: nothing fixed)."""
    if fixed is None:
        return None
    a = np.asarray(fixed)
    if a.dtype == bool:
        if a.size != J:
            raise ValueError("fixed_coefficients mask must have one entry per column")
        a = np.flatnonzero(a)
    a = np.ascontiguousarray(a, np.int32)
    return a if a.size else None


def fit_cyclops_model(data, prior: Optional[PriorSpec] = None, control: Optional[ControlSpec] = None,
                      weights=None, starting_coefficients=None, device: int = 0,
                      host_loop: bool = False, fixed_coefficients=None) -> FitResult:
    """fitCyclopsModel (R/ModelFit.R:65): one fit, CCD loop on the GPU.

    ``fixed_coefficients`` (a boolean mask over the columns, or column ids)
    holds those coefficients at their starting values, as the reference's
    fixedCoefficients does.  ``host_loop=True`` runs the plain FP64
    single-fit GPU CCD instead: the host drives the engine coordinate by
    coordinate, reading (gradient, Hessian) back each time, as the
    reference's CyclicCoordinateDescent does."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    prior = prior or create_prior("none")
    control = control or create_control()
    p, keep_ex = _prior_struct(ds.data, prior)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    s = None if starting_coefficients is None else np.ascontiguousarray(starting_coefficients, np.float64)
    fx = _fixed_columns(fixed_coefficients, ds.data.J)
    spec = N.FitSpec(weights=_ptr(w), variance=prior.variance, start_beta=_ptr(s), fixed=_ptr(fx),
                     n_fixed=0 if fx is None else int(fx.size))
    beta = np.zeros(ds.data.J)
    out = N.FitResult(beta=beta.ctypes.data)
    c = _control_struct(control)
    fn = N.lib().cyc_fit_host_loop if host_loop else N.lib().cyc_fit
    N.check(fn(ds.handle, C.byref(p), C.byref(spec), C.byref(c), C.byref(out)))
    return FitResult(beta, out.log_likelihood, out.log_prior, out.iterations, out.return_flag)


@dataclasses.dataclass
class ProfileBounds:
    columns: np.ndarray           # the profiled columns
    lower: np.ndarray             # lower confidence bound per column (NaN: no bracket found)
    upper: np.ndarray             # upper confidence bound per column
    evaluations: np.ndarray       # refits spent on both bounds
    fit: FitResult                # the fit the bounds are around


def profile_threshold(level: float = 0.95) -> float:
    """qchisq(level, df = 1) / 2 (R/ModelFit.R:772): z^2 / 2 with z the
    (1 + level) / 2 normal quantile."""
    if not 0.01 <= level <= 0.99:
        raise ValueError("level must be between 0 and 1")
    z = statistics.NormalDist().inv_cdf((1.0 + level) / 2.0)
    return z * z / 2.0


def profile_bounds(data, columns: Sequence[int], prior: Optional[PriorSpec] = None,
                   control: Optional[ControlSpec] = None, level: float = 0.95, threshold: Optional[float] = None,
                   include_penalty: bool = True, override_no_regularization: bool = False, weights=None,
                   starting_coefficients=None, device: int = 0) -> ProfileBounds:
    """confint.cyclopsFit (R/ModelFit.R:762-800) through
    CcdInterface::profileModel with one thread: fit on the GPU, then the
    profile-likelihood bounds of `columns`, each refit on the GPU."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    prior = prior or create_prior("none")
    control = control or create_control()
    thr = profile_threshold(level) if threshold is None else float(threshold)
    p, keep_ex = _prior_struct(ds.data, prior)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    s = None if starting_coefficients is None else np.ascontiguousarray(starting_coefficients, np.float64)
    spec = N.FitSpec(weights=_ptr(w), variance=prior.variance, start_beta=_ptr(s))
    cols = np.ascontiguousarray(columns, np.int32)
    n = int(cols.size)
    lo, up, ev = np.zeros(n), np.zeros(n), np.zeros(n, np.int32)
    beta = np.zeros(ds.data.J)
    out = N.FitResult(beta=beta.ctypes.data)
    c = _control_struct(control)
    N.check(N.lib().cyc_profile_bounds(ds.handle, C.byref(p), C.byref(spec), C.byref(c), _ptr(cols), n, thr,
                                       int(include_penalty), int(override_no_regularization), _ptr(lo), _ptr(up),
                                       _ptr(ev), C.byref(out)))
    return ProfileBounds(cols, lo, up, ev, FitResult(beta, out.log_likelihood, out.log_prior, out.iterations,
                                                     out.return_flag))


def profile_log_likelihood(data, column: int, points: Sequence[float], prior: Optional[PriorSpec] = None,
                           control: Optional[ControlSpec] = None, include_penalty: bool = True, weights=None,
                           starting_coefficients=None, device: int = 0, batched: bool = False) -> np.ndarray:
    """getCyclopsProfileLogLikelihood (R/ModelFit.R:816-826) through
    CcdInterface::evaluateProfileModel with one thread: fit on the GPU,
    then the profile log likelihood of `column` at each point.

    ``batched=True`` refits all points together in the persistent batch
    kernel, each from the mode (``starting_coefficients``, or fitted first
    when None); values then agree with the one-thread order to the
    convergence tolerance."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    prior = prior or create_prior("none")
    control = control or create_control()
    p, keep_ex = _prior_struct(ds.data, prior)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    s = None if starting_coefficients is None else np.ascontiguousarray(starting_coefficients, np.float64)
    spec = N.FitSpec(weights=_ptr(w), variance=prior.variance, start_beta=_ptr(s))
    pts = np.ascontiguousarray(points, np.float64)
    vals = np.zeros(pts.size)
    c = _control_struct(control)
    fn = N.lib().cyc_profile_log_likelihood_batch if batched else N.lib().cyc_profile_log_likelihood
    N.check(fn(ds.handle, C.byref(p), C.byref(spec), C.byref(c), int(column), _ptr(pts), int(pts.size),
               int(include_penalty), _ptr(vals)))
    return vals


@dataclasses.dataclass
class CvAutoResult:
    variance: float               # the variance the search settles on
    expected: float               # the search's predicted held-out log likelihood there
    tried: np.ndarray             # (steps, 3): variance, mean, stdev of each step


def cv_auto_search(data, prior: PriorSpec, fold_of_row, n_folds: int, starting_variance: float = -1.0,
                   control: Optional[ControlSpec] = None, device: int = 0, weights=None) -> CvAutoResult:
    """Auto-search cross-validation (createControl(cvType = "auto"), R's
    default; AutoSearchCrossValidationDriver): one variance per step, every
    fold refit on the GPU as one batched solve, the next variance proposed by
    the reference's unimodal search.  `fold_of_row`: K fold ids, or
    (repetitions, K); `weights`: K observation weights (as cv_grid_fit)."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    control = control or create_control()
    p, keep_ex = _prior_struct(ds.data, prior)
    folds = np.ascontiguousarray(np.atleast_2d(fold_of_row), np.int32)
    n_reps = folds.shape[0]
    bv, val, n = C.c_double(), C.c_double(), C.c_int()
    tv, tm, ts = np.zeros(64), np.zeros(64), np.zeros(64)
    c = _control_struct(control)
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    N.check(N.lib().cyc_cv_auto_search(ds.handle, C.byref(p), _ptr(folds), int(n_folds), int(n_reps), _ptr(w),
                                       float(starting_variance), C.byref(c), C.byref(bv), C.byref(val), _ptr(tv),
                                       _ptr(tm), _ptr(ts), 64, C.byref(n)))
    k = min(n.value, 64)
    return CvAutoResult(bv.value, val.value, np.stack([tv[:k], tm[:k], ts[:k]], axis=1))


@dataclasses.dataclass
class AsymptoticVariance:
    columns: np.ndarray           # the columns with a row / column in the matrices
    fisher: np.ndarray            # Fisher information (precision) matrix
    variance: np.ndarray          # its inverse
    standard_errors: np.ndarray   # sqrt of the variance diagonal


def asymptotic_variance(data, beta, prior: PriorSpec, device: int = 0) -> AsymptoticVariance:
    """getAsymptoticVariance (CyclicCoordinateDescent.cpp:1249-1352): the
    Fisher information over the columns that are not fixed and, under a
    Laplace prior, not at zero, computed on the GPU at `beta`; its inverse
    (the reference inverts with Eigen on the host, as here)."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    b = np.ascontiguousarray(beta, np.float64)
    cols = [j for j in range(ds.data.J)
            if not (ds.data.has_offset and j == 0) and (prior.prior_type != PRIOR_LAPLACE or b[j] != 0.0)]
    eng = Engine(ds)
    eng.compute_xbeta(b)
    eng.compute_remaining_statistics()
    fisher = eng.fisher_information(cols)
    var = np.linalg.inv(fisher) if len(cols) else np.zeros((0, 0))
    return AsymptoticVariance(np.asarray(cols, np.int32), fisher, var, np.sqrt(np.diag(var)))


def launch_count() -> int:
    """Kernels launched by libcyclops_b200.so in this process."""
    return int(N.lib().cyc_launch_count())


def batch_fit(data, prior: PriorSpec, variances: Sequence[float], weights: Optional[Sequence] = None,
              control: Optional[ControlSpec] = None, starts=None, device: int = 0,
              fixed_coefficients=None) -> List[FitResult]:
    """F fits sharing one dataset, advanced together on the GPU.  `weights` is
    a list of K-vectors (or None entries) or a (F, K) array;
    `fixed_coefficients` (mask or ids) holds the same columns fixed in every
    fit, at each fit's starting values."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    control = control or create_control()
    F = len(variances)
    p, keep_ex = _prior_struct(ds.data, prior)
    fx = _fixed_columns(fixed_coefficients, ds.data.J)
    specs = (N.FitSpec * F)()
    results = (N.FitResult * F)()
    keep = []
    betas = np.zeros((F, ds.data.J))
    for f in range(F):
        w = None
        if weights is not None and weights[f] is not None:
            w = np.ascontiguousarray(weights[f], np.float64)
            keep.append(w)
        s = None
        if starts is not None and starts[f] is not None:
            s = np.ascontiguousarray(starts[f], np.float64)
            keep.append(s)
        specs[f] = N.FitSpec(weights=_ptr(w), variance=float(variances[f]), start_beta=_ptr(s), fixed=_ptr(fx),
                             n_fixed=0 if fx is None else int(fx.size))
        results[f] = N.FitResult(beta=betas[f].ctypes.data)
    c = _control_struct(control)
    N.check(N.lib().cyc_batch_fit(ds.handle, C.byref(p), specs, F, C.byref(c), results))
    return [FitResult(betas[f].copy(), results[f].log_likelihood, results[f].log_prior,
                      results[f].iterations, results[f].return_flag) for f in range(F)]


@dataclasses.dataclass
class CvGridResult:
    fits: List[FitResult]          # n_var * n_folds, variance-major
    pred_loglik: np.ndarray        # held-out predictive log likelihood per fit
    grid_mean: np.ndarray          # per variance: mean over folds (NaN ignored)
    variances: np.ndarray
    best: int                      # index of the variance with the largest mean


def cv_grid_fit(data, prior: PriorSpec, fold_of_row, n_folds: int, variances: Sequence[float],
                control: Optional[ControlSpec] = None, device: int = 0, weights=None) -> CvGridResult:
    """Cross-validation over a prior-variance grid as one batched GPU solve
    (GridSearchCrossValidationDriver + AbstractCrossValidationDriver).
    `weights` (K observation weights) trains each fold at those weights and
    scores the held-out rows at theirs, as the reference's selector does
    with the fit's weights."""
    ds = data if isinstance(data, Dataset) else Dataset(data, device)
    control = control or create_control()
    p, keep_ex = _prior_struct(ds.data, prior)
    fold = np.ascontiguousarray(fold_of_row, np.int32)
    var = np.ascontiguousarray(variances, np.float64)
    F = n_folds * var.size
    results = (N.FitResult * F)()
    betas = np.zeros((F, ds.data.J))
    for f in range(F):
        results[f] = N.FitResult(beta=betas[f].ctypes.data)
    pll = np.zeros(F)
    gm = np.zeros(var.size)
    c = _control_struct(control)
    if weights is None:
        N.check(N.lib().cyc_cv_grid_fit(ds.handle, C.byref(p), _ptr(fold), int(n_folds), _ptr(var), int(var.size),
                                        C.byref(c), results, _ptr(pll), _ptr(gm)))
    else:
        w = np.ascontiguousarray(weights, np.float64)
        N.check(N.lib().cyc_cv_grid_fit_weighted(ds.handle, C.byref(p), _ptr(fold), int(n_folds), _ptr(w), _ptr(var),
                                                 int(var.size), C.byref(c), results, _ptr(pll), _ptr(gm)))
    fits = [FitResult(betas[f].copy(), results[f].log_likelihood, results[f].log_prior,
                      results[f].iterations, results[f].return_flag) for f in range(F)]
    best = int(np.nanargmax(gm)) if np.any(np.isfinite(gm)) else -1
    return CvGridResult(fits, pll, gm, var, best)


def fold_ids_from_weights(masks: np.ndarray) -> np.ndarray:
    """(folds, K) 0/1 masks that partition the rows -> fold id per row."""
    held = masks == 0
    if not np.all(held.sum(axis=0) == 1):
        raise ValueError("masks must hold out every row exactly once")
    return np.argmax(held, axis=0).astype(np.int32)


def cv_fold_weights(K: int, folds: int, seed: int, ids=None, n_reps: int = 1) -> np.ndarray:
    """(n_reps*folds, K) 0/1 masks, by row (ids None) or by stratum id, drawn
    exactly as the reference's CrossValidationSelector draws them."""
    out = np.zeros((n_reps * folds, K))
    idv = None if ids is None else np.ascontiguousarray(ids, np.int32)
    N.check(N.lib().cyc_cv_fold_weights(int(K), _ptr(idv), int(folds), int(seed), int(ids is None),
                                        int(n_reps), _ptr(out)))
    return out


def bootstrap_weights(K: int, n_replicates: int, seed: int, ids=None, unit_exclude=None) -> np.ndarray:
    """(n_replicates, K) bootstrap weights drawn exactly as the reference's
    BootstrapSelector draws them for BootstrapDriver: each replicate resamples
    the units (`ids`, one per row by default) with replacement; a row's
    weight is its unit's draw count.  Fit the replicates together with
    batch_fit(data, prior, [variance] * n_replicates, weights).  The
    reference's driver warm-starts each replicate from the previous one's
    coefficients; batch_fit starts every replicate from `starts` (zero by
    default), so fits agree with the driver's to the convergence tolerance."""
    out = np.zeros((n_replicates, K))
    idv = None if ids is None else np.ascontiguousarray(ids, np.int32)
    ex = None if unit_exclude is None else np.ascontiguousarray(unit_exclude, np.float64)
    N.check(N.lib().cyc_bootstrap_weights(int(K), _ptr(idv), int(n_replicates), int(seed), _ptr(ex), _ptr(out)))
    return out


def last_run_stats() -> dict:
    s = N.RunStats()
    N.check(N.lib().cyc_last_run_stats(C.byref(s)))
    out = {}
    for k, _ in N.RunStats._fields_:
        v = getattr(s, k)
        out[k] = list(v) if hasattr(v, "__len__") else v
    return out

"""TEST INFRASTRUCTURE: ctypes access to the two CPU oracles.

* ``ref``  -- oracle/_ref/libcyclops_ref.so: the reference Cyclops engine
  compiled from its own sources (oracle/Makefile) driven by ref_harness.cpp.
* ``port`` -- oracle/_ref/libccd_oracle.so: the plain-C restatement
  (oracle/ccd_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
module.  Nothing in the product package does.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


class Problem(C.Structure):
    _fields_ = [
        ("model", C.c_int), ("K", C.c_int), ("J", C.c_int),
        ("pid", C.c_void_p), ("y", C.c_void_p), ("time", C.c_void_p),
        ("col_format", C.c_void_p), ("col_ptr", C.c_void_p), ("col_idx", C.c_void_p),
        ("val_ptr", C.c_void_p), ("col_val", C.c_void_p),
        ("has_offset", C.c_int), ("has_intercept", C.c_int),
        ("prior_type", C.c_int), ("variance", C.c_double),
        ("exclude", C.c_void_p), ("n_exclude", C.c_int),
        ("weights", C.c_void_p),
        ("fixed", C.c_void_p), ("n_fixed", C.c_int),
    ]


class Control(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double), ("max_iterations", C.c_int),
        ("convergence_type", C.c_int), ("use_kkt_swindle", C.c_int),
        ("initial_bound", C.c_double), ("max_bound_count", C.c_int),
    ]


class Result(C.Structure):
    _fields_ = [
        ("beta", C.c_void_p), ("log_likelihood", C.c_double), ("log_prior", C.c_double),
        ("iterations", C.c_int), ("return_flag", C.c_int),
    ]


@dataclasses.dataclass
class Fit:
    beta: np.ndarray
    log_likelihood: float
    log_prior: float
    iterations: int
    return_flag: int


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def make_problem(data, prior_type=1, variance=1.0, exclude=None, weights=None, fixed=None):
    """Returns (Problem, keepalive) for a cyclops_b200.data.CyclopsData;
    `fixed`: columns held at their start values."""
    if exclude is None:
        exclude = [1 if data.has_offset else 0] if data.has_intercept else []
    keep = {
        "pid": None if data.pid is None else np.ascontiguousarray(data.pid, np.int32),
        "y": np.ascontiguousarray(data.y, np.float64),
        "time": None if data.time is None else np.ascontiguousarray(data.time, np.float64),
        "fmt": np.ascontiguousarray(data.col_format, np.int32),
        "cp": np.ascontiguousarray(data.col_ptr, np.int64),
        "ci": np.ascontiguousarray(data.col_idx, np.int32),
        "vp": np.ascontiguousarray(data.val_ptr, np.int64),
        "cv": np.ascontiguousarray(data.col_val, np.float64),
        "ex": np.ascontiguousarray(exclude, np.int32),
        "w": None if weights is None else np.ascontiguousarray(weights, np.float64),
        "fx": None if not fixed else np.ascontiguousarray(fixed, np.int32),
    }
    p = Problem(
        model=data.model, K=data.K, J=data.J, pid=_ptr(keep["pid"]), y=_ptr(keep["y"]),
        time=_ptr(keep["time"]), col_format=_ptr(keep["fmt"]), col_ptr=_ptr(keep["cp"]),
        col_idx=_ptr(keep["ci"]), val_ptr=_ptr(keep["vp"]), col_val=_ptr(keep["cv"]),
        has_offset=int(data.has_offset), has_intercept=int(data.has_intercept),
        prior_type=prior_type, variance=variance, exclude=_ptr(keep["ex"]),
        n_exclude=len(exclude), weights=_ptr(keep["w"]), fixed=_ptr(keep["fx"]),
        n_fixed=0 if keep["fx"] is None else int(keep["fx"].size))
    return p, keep


def make_control(tolerance=1e-6, max_iterations=1000, convergence_type=0, use_kkt_swindle=0,
                 initial_bound=2.0, max_bound_count=5) -> Control:
    """Defaults are the reference's ModeFindingArguments (src/cyclops/CcdInterface.h:70-94)."""
    return Control(tolerance=tolerance, max_iterations=max_iterations,
                   convergence_type=convergence_type, use_kkt_swindle=use_kkt_swindle,
                   initial_bound=initial_bound, max_bound_count=max_bound_count)


def build(quiet: bool = True) -> None:
    """Build the oracle libraries (the reference engine only where its sources exist)."""
    cmd = ["make", "-C", HERE, "-j8"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


class _Lib:
    def __init__(self, name, prefix):
        path = os.path.join(REF_DIR, name)
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        self.prefix = prefix
        le = getattr(self.lib, prefix + "last_error")
        le.restype = C.c_char_p
        self._last_error = le
        P, V = C.POINTER, C.c_void_p
        sigs = {
            "fit": [P(Problem), P(Control), V, P(Result)],
            "engine_probe" if prefix == "ref_" else "probe": [P(Problem), V, V, V, V, P(C.c_double)],
            "predictive_loglik": [P(Problem), V, V, P(C.c_double)],
        }
        if prefix == "ref_":
            sigs["cv_weights"] = [C.c_int, V, C.c_int, C.c_long, C.c_int, C.c_int, V]
            sigs["fisher"] = [P(Problem), V, V, C.c_int, V, C.c_int]
            sigs["predictive_estimates"] = [P(Problem), V, V, V]
            sigs["cv_grid"] = [P(Problem), P(Control), C.c_int, C.c_long, C.c_int, C.c_double, C.c_double, C.c_int,
                               C.c_int, V, V, V]
            sigs["cv_auto"] = [P(Problem), P(Control), C.c_int, C.c_int, C.c_long, C.c_int, C.c_double, C.c_int,
                               P(C.c_double), P(C.c_double), V, V, V, C.c_int, P(C.c_int)]
            sigs["fit_device"] = [P(Problem), P(Control), V, P(Result), C.c_int]
            sigs["profile"] = [P(Problem), P(Control), V, V, C.c_int, C.c_double, C.c_int, C.c_int, V, V, V,
                               P(Result), C.c_int]
            sigs["profile_points"] = [P(Problem), P(Control), V, C.c_int, V, C.c_int, C.c_int, V, C.c_int]
        else:
            sigs["profile_points"] = [P(Problem), P(Control), V, C.c_int, V, C.c_int, C.c_int, V]
            sigs["profile"] = [P(Problem), P(Control), V, V, C.c_int, C.c_double, C.c_int, C.c_int, V, V, V,
                               P(Result)]
        for name, args in sigs.items():
            fn = getattr(self.lib, prefix + name, None)
            if fn is not None:
                fn.argtypes = args
                fn.restype = C.c_int

    def err(self) -> str:
        return self._last_error().decode()

    def fit(self, data, prior_type=1, variance=1.0, control: Optional[Control] = None,
            exclude=None, weights=None, start=None, fixed=None) -> Fit:
        p, keep = make_problem(data, prior_type, variance, exclude, weights, fixed)
        c = control or make_control()
        beta = np.zeros(data.J)
        r = Result(beta=beta.ctypes.data)
        s = None if start is None else np.ascontiguousarray(start, np.float64)
        rc = getattr(self.lib, self.prefix + "fit")(C.byref(p), C.byref(c), _ptr(s), C.byref(r))
        if rc:
            raise RuntimeError(self.err())
        return Fit(beta, r.log_likelihood, r.log_prior, r.iterations, r.return_flag)

    def probe(self, data, beta, prior_type=1, variance=1.0, exclude=None, weights=None):
        p, keep = make_problem(data, prior_type, variance, exclude, weights)
        b = np.ascontiguousarray(beta, np.float64)
        g = np.zeros(data.J)
        h = np.zeros(data.J)
        xb = np.zeros(data.K)
        ll = C.c_double()
        fn = getattr(self.lib, self.prefix + ("engine_probe" if self.prefix == "ref_" else "probe"))
        rc = fn(C.byref(p), _ptr(b), _ptr(g), _ptr(h), _ptr(xb), C.byref(ll))
        if rc:
            raise RuntimeError(self.err())
        return g, h, xb, ll.value

    def fisher(self, data, beta, columns, device=0):
        """CyclicCoordinateDescent::computeFisherInformation at `beta` (n x n)."""
        p, keep = make_problem(data, 1, 1.0, None, None)
        b = np.ascontiguousarray(beta, np.float64)
        cols = np.ascontiguousarray(columns, np.int32)
        out = np.zeros((cols.size, cols.size))
        rc = self.lib.ref_fisher(C.byref(p), _ptr(b), _ptr(cols), int(cols.size), _ptr(out), int(device))
        if rc:
            raise RuntimeError(self.err())
        return out

    def profile(self, data, columns, prior_type=1, variance=1.0, threshold=1.920729, include_penalty=True,
                override_no_regularization=False, control: Optional[Control] = None, exclude=None,
                weights=None, start=None, device=0):
        """CcdInterface::profileModel with one thread: fit, then each column's
        (lower, upper) profile bound and the refits both took.  Returns
        (lower, upper, evaluations, Fit)."""
        p, keep = make_problem(data, prior_type, variance, exclude, weights)
        c = control or make_control()
        cols = np.ascontiguousarray(columns, np.int32)
        n = int(cols.size)
        lo, up, ev = np.zeros(n), np.zeros(n), np.zeros(n, np.int32)
        beta = np.zeros(data.J)
        r = Result(beta=beta.ctypes.data)
        s = None if start is None else np.ascontiguousarray(start, np.float64)
        args = [C.byref(p), C.byref(c), _ptr(s), _ptr(cols), n, float(threshold), int(include_penalty),
                int(override_no_regularization), _ptr(lo), _ptr(up), _ptr(ev), C.byref(r)]
        if self.prefix == "ref_":
            args.append(int(device))
        if getattr(self.lib, self.prefix + "profile")(*args):
            raise RuntimeError(self.err())
        return lo, up, ev, Fit(beta, r.log_likelihood, r.log_prior, r.iterations, r.return_flag)

    def profile_points(self, data, column, points, prior_type=1, variance=1.0, include_penalty=True,
                       control: Optional[Control] = None, exclude=None, weights=None, start=None, device=0):
        """CcdInterface::evaluateProfileModel with one thread: the profile log
        likelihood (+ log prior) of `column` at each of `points`."""
        p, keep = make_problem(data, prior_type, variance, exclude, weights)
        c = control or make_control()
        pts = np.ascontiguousarray(points, np.float64)
        vals = np.zeros(pts.size)
        s = None if start is None else np.ascontiguousarray(start, np.float64)
        args = [C.byref(p), C.byref(c), _ptr(s), int(column), _ptr(pts), int(pts.size), int(include_penalty),
                _ptr(vals)]
        if self.prefix == "ref_":
            args.append(int(device))
        if getattr(self.lib, self.prefix + "profile_points")(*args):
            raise RuntimeError(self.err())
        return vals

    def predictive_estimates(self, data, beta, weights=None, fill=0.0):
        """getPredictiveEstimates at `beta` (rows with zero weight keep `fill`)."""
        p, keep = make_problem(data, 1, 1.0, None, None)
        b = np.ascontiguousarray(beta, np.float64)
        w = None if weights is None else np.ascontiguousarray(weights, np.float64)
        y = np.full(data.K, float(fill))
        if self.lib.ref_predictive_estimates(C.byref(p), _ptr(b), _ptr(w), _ptr(y)):
            raise RuntimeError(self.err())
        return y

    def cv_auto(self, data, prior_type, fold=10, n_reps=1, seed=123, by_row=True, starting_variance=-1.0,
                reset_coefficients=True, control: Optional[Control] = None, exclude=None):
        """AutoSearchCrossValidationDriver run by the reference (one thread).
        Returns (best_variance, best_value, tried) with tried an (n, 3) array
        of (variance, mean, stdev) as the driver logged them."""
        p, keep = make_problem(data, prior_type, 1.0, exclude, None)
        c = control or make_control()
        bv, bval, n = C.c_double(), C.c_double(), C.c_int()
        tv, tm, ts = np.zeros(64), np.zeros(64), np.zeros(64)
        rc = ref_dyn().lib.ref_cv_auto(C.byref(p), C.byref(c), int(fold), int(n_reps), int(seed), int(by_row),
                                  float(starting_variance), int(reset_coefficients), C.byref(bv), C.byref(bval),
                                  _ptr(tv), _ptr(tm), _ptr(ts), 64, C.byref(n))
        if rc:
            raise RuntimeError(ref_dyn().err())
        k = n.value
        return bv.value, bval.value, np.stack([tv[:k], tm[:k], ts[:k]], axis=1)

    def cv_grid(self, data, prior_type, fold=10, seed=123, by_row=True, lower=0.01, upper=20.0, grid_steps=10,
                reset_coefficients=True, control: Optional[Control] = None, exclude=None, weights=None):
        """GridSearchCrossValidationDriver run by the reference (one thread),
        with `weights` as the fit's weights.  Returns (points, values,
        fold_pred[grid_steps, fold])."""
        p, keep = make_problem(data, prior_type, 1.0, exclude, weights)
        c = control or make_control()
        pts, vals = np.zeros(grid_steps), np.zeros(grid_steps)
        fp = np.full(grid_steps * fold, np.nan)
        rc = ref_dyn().lib.ref_cv_grid(C.byref(p), C.byref(c), int(fold), int(seed), int(by_row), float(lower),
                                       float(upper), int(grid_steps), int(reset_coefficients), _ptr(pts), _ptr(vals),
                                       _ptr(fp))
        if rc:
            raise RuntimeError(ref_dyn().err())
        return pts, vals, fp.reshape(grid_steps, fold)

    def predictive_loglik(self, data, beta, held_out, weights=None):
        p, keep = make_problem(data, 1, 1.0, None, weights)
        b = np.ascontiguousarray(beta, np.float64)
        w = np.ascontiguousarray(held_out, np.float64)
        out = C.c_double()
        rc = getattr(self.lib, self.prefix + "predictive_loglik")(C.byref(p), _ptr(b), _ptr(w),
                                                                   C.byref(out))
        if rc:
            raise RuntimeError(self.err())
        return out.value


_cache = {}


def ref() -> _Lib:
    """The reference engine (raises if it cannot be built here)."""
    if "ref" not in _cache:
        _cache["ref"] = _Lib("libcyclops_ref.so", "ref_")
    return _cache["ref"]


def ref_dyn() -> _Lib:
    """The reference engine linked against the process's shared C++ runtime
    (for the CV drivers, whose logging formats numbers through iostreams)."""
    if "ref_dyn" not in _cache:
        _cache["ref_dyn"] = _Lib("libcyclops_ref_dyn.so", "ref_")
    return _cache["ref_dyn"]


def port() -> _Lib:
    """The plain-C restatement."""
    if "port" not in _cache:
        _cache["port"] = _Lib("libccd_oracle.so", "ccd_oracle_")
    return _cache["port"]


def have_ref() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libcyclops_ref.so"))


_CV_SCRIPT = r"""
import ctypes as C, sys, struct
L = C.CDLL(sys.argv[1])
f = L.ref_cv_weights
f.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_long, C.c_int, C.c_int, C.c_void_p]
K, fold, seed, by_row, reps = map(int, sys.argv[2:7])
raw = sys.stdin.buffer.read()
ids = (C.c_int * K).from_buffer_copy(raw)
out = (C.c_double * (K * fold * reps))()
rc = f(K, C.addressof(ids), fold, seed, by_row, reps, C.addressof(out))
if rc:
    sys.exit(3)
sys.stdout.buffer.write(bytes(out))
"""


def ref_cv_weights(K, ids, fold, seed, by_row=True, n_reps=1) -> np.ndarray:
    """Fold masks from the reference's CrossValidationSelector.

    Runs in a child interpreter that loads the reference library before
    numpy: the selector's logging path crashes when numpy's C++ runtime
    was loaded first into the same process."""
    path = os.path.join(REF_DIR, "libcyclops_ref.so")
    if not os.path.exists(path):
        build()
    ids = np.ascontiguousarray(ids, np.int32)
    import sys
    p = subprocess.run([sys.executable, "-c", _CV_SCRIPT, path, str(K), str(fold), str(seed),
                        str(int(by_row)), str(n_reps)], input=ids.tobytes(), capture_output=True,
                       check=True)
    return np.frombuffer(p.stdout, dtype=np.float64).reshape(n_reps * fold, K).copy()


_BOOT_SCRIPT = r"""
import ctypes as C, sys
L = C.CDLL(sys.argv[1])
f = L.ref_bootstrap_weights
f.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_long, C.c_void_p]
K, reps, seed = map(int, sys.argv[2:5])
raw = sys.stdin.buffer.read()
ids = (C.c_int * K).from_buffer_copy(raw)
out = (C.c_double * (K * reps))()
if f(K, C.addressof(ids), reps, seed, C.addressof(out)):
    sys.exit(3)
sys.stdout.buffer.write(bytes(out))
"""


def ref_bootstrap_weights(K, ids, n_replicates, seed) -> np.ndarray:
    """Replicate weights from the reference's BootstrapSelector (by unit id,
    one permute per replicate as BootstrapDriver does), in a child
    interpreter for the same reason as ref_cv_weights."""
    path = os.path.join(REF_DIR, "libcyclops_ref.so")
    if not os.path.exists(path):
        build()
    ids = np.ascontiguousarray(ids, np.int32)
    import sys
    p = subprocess.run([sys.executable, "-c", _BOOT_SCRIPT, path, str(K), str(n_replicates), str(seed)],
                       input=ids.tobytes(), capture_output=True, check=True)
    return np.frombuffer(p.stdout, dtype=np.float64).reshape(n_replicates, K).copy()


class IngestInput(C.Structure):
    _fields_ = [("model", C.c_int), ("n_outcomes", C.c_longlong), ("stratum_id", C.c_void_p),
                ("row_id", C.c_void_p), ("y", C.c_void_p), ("time", C.c_void_p),
                ("n_covariates", C.c_longlong), ("covariate_id", C.c_void_p), ("covariate_row", C.c_void_p),
                ("covariate_value", C.c_void_p), ("add_intercept", C.c_int), ("offset_from_time", C.c_int)]


class IngestOutput(C.Structure):
    _fields_ = [("K", C.c_int), ("J", C.c_int), ("col_format", C.POINTER(C.c_int)),
                ("col_ptr", C.POINTER(C.c_longlong)), ("col_idx", C.POINTER(C.c_int)),
                ("val_ptr", C.POINTER(C.c_longlong)), ("col_val", C.POINTER(C.c_double)),
                ("col_label", C.POINTER(C.c_longlong)), ("pid", C.POINTER(C.c_int)),
                ("y", C.POINTER(C.c_double)), ("time", C.POINTER(C.c_double)),
                ("has_offset", C.c_int), ("has_intercept", C.c_int)]


_INGEST_SCRIPT = r"""
import ctypes as C, sys, struct
L = C.CDLL(sys.argv[1])
class IngestInput(C.Structure):
    _fields_ = [("model", C.c_int), ("n_outcomes", C.c_longlong), ("stratum_id", C.c_void_p),
                ("row_id", C.c_void_p), ("y", C.c_void_p), ("time", C.c_void_p),
                ("n_covariates", C.c_longlong), ("covariate_id", C.c_void_p), ("covariate_row", C.c_void_p),
                ("covariate_value", C.c_void_p), ("add_intercept", C.c_int), ("offset_from_time", C.c_int)]
class IngestOutput(C.Structure):
    _fields_ = [("K", C.c_int), ("J", C.c_int), ("col_format", C.POINTER(C.c_int)),
                ("col_ptr", C.POINTER(C.c_longlong)), ("col_idx", C.POINTER(C.c_int)),
                ("val_ptr", C.POINTER(C.c_longlong)), ("col_val", C.POINTER(C.c_double)),
                ("col_label", C.POINTER(C.c_longlong)), ("pid", C.POINTER(C.c_int)),
                ("y", C.POINTER(C.c_double)), ("time", C.POINTER(C.c_double)),
                ("has_offset", C.c_int), ("has_intercept", C.c_int)]
raw = sys.stdin.buffer.read()
model, n, m, hs, ht, hv, ai, off = struct.unpack_from("<iqqiiiii", raw, 0)
pos = struct.calcsize("<iqqiiiii")
def take(count, ctype):
    global pos
    size = count * C.sizeof(ctype)
    buf = (ctype * max(count, 1)).from_buffer_copy(raw[pos:pos + size] + bytes(C.sizeof(ctype)))
    pos += size
    return buf
st = take(n, C.c_longlong) if hs else None
row = take(n, C.c_longlong); y = take(n, C.c_double)
tm = take(n, C.c_double) if ht else None
cid = take(m, C.c_longlong); crow = take(m, C.c_longlong)
cv = take(m, C.c_double) if hv else None
a = lambda b: C.addressof(b) if b is not None else None
inp = IngestInput(model, n, a(st), a(row), a(y), a(tm), m, a(cid), a(crow), a(cv), ai, off)
out = IngestOutput()
L.ref_ingest.argtypes = [C.POINTER(IngestInput), C.POINTER(IngestOutput)]
L.ref_last_error.restype = C.c_char_p
if L.ref_ingest(C.byref(inp), C.byref(out)):
    sys.stderr.write(L.ref_last_error().decode())
    sys.exit(3)
J, K = out.J, out.K
ni, nv = out.col_ptr[J], out.val_ptr[J]
w = sys.stdout.buffer
w.write(struct.pack("<iiiiiqq", K, J, 1 if out.time else 0, out.has_offset, out.has_intercept, ni, nv))
def put(ptr, count, ctype):
    w.write(C.string_at(ptr, count * C.sizeof(ctype)) if count else b"")
put(out.col_format, J, C.c_int); put(out.col_ptr, J + 1, C.c_longlong); put(out.col_idx, ni, C.c_int)
put(out.val_ptr, J + 1, C.c_longlong); put(out.col_val, nv, C.c_double); put(out.col_label, J, C.c_longlong)
put(out.pid, K, C.c_int); put(out.y, K, C.c_double)
if out.time:
    put(out.time, K, C.c_double)
"""


def ref_ingest(model, outcomes, covariates, add_intercept, offset_from_time) -> dict:
    """The reference's ModelData loader (loadY, intercept loadX, loadMultipleX,
    the Poisson offset) on tables already in the reference's sort order.

    Runs in a child interpreter without numpy, for the reason given at
    ref_cv_weights (loadY formats row labels through a stringstream)."""
    import struct
    import sys
    path = os.path.join(REF_DIR, "libcyclops_ref.so")
    if not os.path.exists(path):
        build()
    st, tm, cv = outcomes.get("stratumId"), outcomes.get("time"), covariates.get("covariateValue")
    n, m = len(outcomes["rowId"]), len(covariates["rowId"])
    parts = [struct.pack("<iqqiiiii", model, n, m, st is not None, tm is not None, cv is not None,
                         int(add_intercept), int(offset_from_time))]
    if st is not None:
        parts.append(np.ascontiguousarray(st, np.int64).tobytes())
    parts += [np.ascontiguousarray(outcomes["rowId"], np.int64).tobytes(),
              np.ascontiguousarray(outcomes["y"], np.float64).tobytes()]
    if tm is not None:
        parts.append(np.ascontiguousarray(tm, np.float64).tobytes())
    parts += [np.ascontiguousarray(covariates["covariateId"], np.int64).tobytes(),
              np.ascontiguousarray(covariates["rowId"], np.int64).tobytes()]
    if cv is not None:
        parts.append(np.ascontiguousarray(cv, np.float64).tobytes())
    p = subprocess.run([sys.executable, "-c", _INGEST_SCRIPT, path], input=b"".join(parts), capture_output=True)
    if p.returncode:
        raise RuntimeError(p.stderr.decode(errors="replace")[-500:])
    buf = p.stdout
    K, J, ht, hoff, hint, ni, nv = struct.unpack_from("<iiiiiqq", buf, 0)
    pos = struct.calcsize("<iiiiiqq")

    def take(count, dt):
        nonlocal pos
        a = np.frombuffer(buf, dtype=dt, count=count, offset=pos).copy()
        pos += count * np.dtype(dt).itemsize
        return a

    res = {"col_format": take(J, np.int32), "col_ptr": take(J + 1, np.int64), "col_idx": take(ni, np.int32),
           "val_ptr": take(J + 1, np.int64), "col_val": take(nv, np.float64), "col_label": take(J, np.int64),
           "pid": take(K, np.int32), "y": take(K, np.float64)}
    res["time"] = take(K, np.float64) if ht else None
    res["has_offset"], res["has_intercept"] = hoff, hint
    return res

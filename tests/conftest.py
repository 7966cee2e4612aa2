import glob
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from cyclops_b200 import data as D  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def golden_names():
    """The plain fit fixtures (not the CV folds, ingest tables or swindle fits)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not p.endswith(("cv_folds.npz", "bootstrap_weights.npz"))
                  and not os.path.basename(p).startswith(("ingest_", "swindle_", "profile_", "small_", "cvauto_")))


def small_names():
    """Tiny designs from the reference's own tests (test-smallCox.R,
    test-smallBernoulli.R, test-smallPoisson.R) with the reference's fits and
    an independent Newton MLE."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "small_*.npz")))


def cvauto_names():
    """The reference's auto-search CV results on fit fixtures' data."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "cvauto_*.npz")))


def profile_names():
    """Profile-likelihood bound fixtures (profileModel)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "profile_*.npz")))


def swindle_names():
    """Fits made with the KKT swindle (useKktSwindle)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "swindle_*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    pid = z["pid"] if z["pid"].size else None
    time = z["time"] if z["time"].size else None
    data = D.CyclopsData(model=int(z["model"]), y=z["y"], col_format=z["col_format"], col_ptr=z["col_ptr"],
                         col_idx=z["col_idx"], val_ptr=z["val_ptr"], col_val=z["col_val"], pid=pid,
                         time=time, has_offset=bool(z["has_offset"]), has_intercept=bool(z["has_intercept"]))
    spec = {k: z[k] for k in z.files}
    spec["weights"] = z["weights"] if z["weights"].size else None
    return data, spec


def exclude_for(data):
    return [1 if data.has_offset else 0] if data.has_intercept else []


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library, built in-tree if missing (fails loudly without nvcc)."""
    from cyclops_b200 import build, _native
    build.build()
    return _native.lib()


def rel_err(a, b, floor=1e-12):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


# The precision contract of an FP64 path against an FP64 oracle run with the
# same prior, variance, tolerance and convergence rule: the same return flag
# and cycle count, the same zero pattern, beta within 1e-6 relative (1e-9
# absolute around zero) and log likelihood within 1e-9 relative.
BETA_RTOL = 1e-6
BETA_ATOL = 1e-9
LL_RTOL = 1e-9


def golden_fit(s):
    """The reference's fit stored in a fixture, as a fit record."""
    return types.SimpleNamespace(beta=np.asarray(s["beta"], float), log_likelihood=float(s["log_likelihood"]),
                                 iterations=int(s["iterations"]), return_flag=int(s["return_flag"]))


def assert_contract(got, want, iterations=True, log_likelihood=True, what="", beta_atol=BETA_ATOL):
    """`got` (beta, log_likelihood, iterations, return_flag) against `want`
    under the precision contract; `iterations=False` drops the cycle count
    (a path whose reported cycles are one phase's), `log_likelihood=False`
    the likelihood (a record that carries none); `beta_atol` widens the
    absolute bound near zero where a test states why."""
    assert got.return_flag == want.return_flag, (what, got.return_flag, want.return_flag)
    if iterations:
        assert got.iterations == want.iterations, (what, got.iterations, want.iterations)
    b, w = np.asarray(got.beta, float), np.asarray(want.beta, float)
    np.testing.assert_array_equal(b != 0, w != 0, err_msg=str(what))
    ok = np.abs(b - w) <= BETA_RTOL * np.abs(w) + beta_atol
    j = int(np.argmin(ok)) if not ok.all() else -1
    assert ok.all(), (what, "column", j, float(b[j]), float(w[j]), "abs", float(abs(b[j] - w[j])))
    if log_likelihood:
        assert rel_err(got.log_likelihood, want.log_likelihood) < LL_RTOL, (what, got.log_likelihood,
                                                                             want.log_likelihood)

import glob
import os
import sys

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
                  if not p.endswith("cv_folds.npz")
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

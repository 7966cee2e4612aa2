"""Auto-search cross-validation on the GPU (cyc_cv_auto_search: every step's
folds one batched solve) against the reference's own
AutoSearchCrossValidationDriver (fixtures tests/golden/cvauto_*.npz)."""
import os

import numpy as np
import pytest

from conftest import ROOT, cvauto_names, exclude_for, load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", cvauto_names())
def test_auto_search_matches_reference(cuda_lib, name):
    from cyclops_b200 import api
    z = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    data, _ = load_golden(str(z["base"]))
    by_row = bool(z["by_row"])
    if by_row:
        ids = np.arange(data.K, dtype=np.int32)
    else:
        pid = np.asarray(data.pid)
        ids = np.concatenate([[0], np.cumsum(pid[1:] != pid[:-1])]).astype(np.int32)
    W = O.ref_cv_weights(data.K, ids, 10, int(z["seed"]), by_row=by_row, n_reps=1)
    fold_of_row = np.argmin(W, axis=0).astype(np.int32)          # the fold that holds each row out
    assert np.all(W[fold_of_row, np.arange(data.K)] == 0)
    prior = api.PriorSpec(int(z["prior"]), 1.0, exclude_for(data))
    res = api.cv_auto_search(data, prior, fold_of_row, 10, float(z["starting_variance"]))
    np.testing.assert_allclose(res.variance, float(z["best_variance"]), rtol=1e-6)
    np.testing.assert_allclose(res.expected, float(z["best_value"]), rtol=1e-6)
    np.testing.assert_allclose(res.tried, z["tried"], rtol=1e-5)

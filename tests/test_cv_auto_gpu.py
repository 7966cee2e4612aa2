"""Auto-search cross-validation on the GPU (cyc_cv_auto_search: every step's
folds one batched solve, Cox folds concurrent single-fit solves) against the
reference's own AutoSearchCrossValidationDriver (fixtures
tests/golden/cvauto_*.npz, a stratified Cox case among them)."""
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


def test_weighted_auto_search_matches_restatement(cuda_lib):
    """Observation weights in the auto search: each step's folds train and
    score at the weights (the selector's original weights)."""
    from cyclops_b200 import api
    from oracle import cv_auto
    data, s = load_golden("lr_laplace_small")
    w = 1.0 + (np.arange(data.K) % 3)
    fold = (np.arange(data.K) * 7 % 5).astype(np.int32)
    W = np.stack([np.where(fold == f, 0.0, w) for f in range(5)])

    def fits(v, train, held_unit):
        f = O.port().fit(data, int(s["prior"]), v, weights=train)
        held = np.where(train == 0, w, 0.0)
        return float("nan") if f.return_flag != 0 else O.port().predictive_loglik(data, f.beta, held, weights=train)

    x, value, trail = cv_auto.auto_search(data, fits, 5, W)
    prior = api.PriorSpec(int(s["prior"]), 1.0, exclude_for(data))
    got = api.cv_auto_search(data, prior, fold, 5, weights=w)
    np.testing.assert_allclose(got.variance, x, rtol=1e-6)
    np.testing.assert_allclose(got.tried, np.array(trail), rtol=1e-6)

"""The batched solver's tuners: a large solve times one cycle at each
candidate cluster size, then at each candidate batch shape (the bound that
splits short, batched columns from long, streamed ones; the rows a batch
may share; its replay levels), keeps the fastest, caches both per problem
shape, and gives the same fits as any fixed size or shape."""
import os

import numpy as np
import pytest

from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu


def _grid(data, fold, n_folds, variances):
    from cyclops_b200 import api
    prior = api.create_prior("laplace", 1.0, exclude=[0])
    return api.cv_grid_fit(data, prior, fold, n_folds, variances, api.create_control(tolerance=1e-8))


def test_tuner_picks_caches_and_matches_fixed_size(cuda_lib, monkeypatch):
    from cyclops_b200 import api
    monkeypatch.delenv("CYC_BATCH_CLUSTER", raising=False)
    d = D.synth_logistic(K=250_000, P=2_500, density=0.005, n_true=40, seed=91)   # ~3.1M entries
    n_folds = 10
    fold = np.random.default_rng(3).integers(0, n_folds, d.K).astype(np.int32)
    variances = [D.laplace_variance(l) for l in (0.3, 1.0, 3.0, 10.0)]       # 40 fits x 3.1M > 1e8
    ds = api.Dataset(d)
    l0 = api.launch_count()
    first = _grid(ds, fold, n_folds, variances)
    l1 = api.launch_count()
    c_first = api.last_run_stats()["cluster_ctas"]
    second = _grid(ds, fold, n_folds, variances)
    l2 = api.launch_count()
    assert c_first in (2, 4, 8)
    assert api.last_run_stats()["cluster_ctas"] == c_first          # cached choice
    assert l2 - l1 < l1 - l0                                          # no probe launches the second time
    for a, b in zip(first.fits, second.fits):
        np.testing.assert_array_equal(a.beta, b.beta)
    monkeypatch.setenv("CYC_BATCH_CLUSTER", "8" if c_first != 8 else "4")
    fixed = _grid(ds, fold, n_folds, variances)
    assert api.last_run_stats()["cluster_ctas"] != c_first
    for a, b in zip(first.fits, fixed.fits):
        assert a.iterations == b.iterations
        np.testing.assert_allclose(a.beta, b.beta, rtol=1e-6, atol=1e-9)


def test_shape_tuner_reports_caches_and_any_shape_gives_the_fits(cuda_lib, monkeypatch):
    """Every batch shape runs the same serial CCD (a batch replays the
    coordinate steps of its columns in order), so the fits agree under the
    precision contract whichever shape the tuner or the caller picks."""
    from cyclops_b200 import api
    from conftest import assert_contract
    monkeypatch.delenv("CYC_BATCH_SHAPE", raising=False)
    monkeypatch.setenv("CYC_BATCH_CLUSTER", "8")
    d = D.synth_logistic(K=250_000, P=2_500, density=0.005, n_true=40, seed=92, zipf=1.1)
    n_folds = 10
    fold = np.random.default_rng(4).integers(0, n_folds, d.K).astype(np.int32)
    variances = [D.laplace_variance(l) for l in (0.3, 1.0, 3.0, 10.0)]
    ds = api.Dataset(d)
    l0 = api.launch_count()
    tuned = _grid(ds, fold, n_folds, variances)
    l1 = api.launch_count()
    st = api.last_run_stats()
    shape = (st["batch_cap"], st["batch_shared_rows"], st["batch_levels"])
    assert shape[0] in (256, 128, 64) and shape[1] in (32, 16) and shape[2] in (8, 2)
    again = _grid(ds, fold, n_folds, variances)
    l2 = api.launch_count()
    assert l2 - l1 < l1 - l0                                          # cached: no probes
    assert (api.last_run_stats()["batch_cap"], api.last_run_stats()["batch_shared_rows"],
            api.last_run_stats()["batch_levels"]) == shape
    for a, b in zip(tuned.fits, again.fits):
        np.testing.assert_array_equal(a.beta, b.beta)
    for forced in ("64,8,1", "256,32,8"):
        monkeypatch.setenv("CYC_BATCH_SHAPE", forced)
        other = _grid(ds, fold, n_folds, variances)
        st = api.last_run_stats()
        assert "%d,%d,%d" % (st["batch_cap"], st["batch_shared_rows"], st["batch_levels"]) == forced
        for i, (a, b) in enumerate(zip(tuned.fits, other.fits)):
            assert_contract(b, a, what=(forced, i))

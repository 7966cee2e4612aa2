"""Cross-validation grids on the device (cyc_cv_grid_fit): folds x prior
variances as one batched solve.  Every fit equals the oracle's fit on the
same training rows, its held-out predictive log likelihood is the oracle's
for its coefficients, and both hold whatever number of CTAs splits the rows
(the cluster size), so the cross-CTA exchange and the batches of short
columns that share rows are covered.

The data mixes an intercept, real-valued sparse columns drawn from a small
pool of rows (so consecutive short columns share rows and batches replay
them serially), and Zipf-sized indicator columns (long columns stream)."""
import os

import numpy as np
import pytest

from conftest import assert_contract, exclude_for, load_golden, rel_err
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu


def _mixed_data(model, K=40_000, n_sparse=120, n_ind=300, seed=5):
    rng = np.random.default_rng(seed)
    b = D.ColumnBuilder(K).intercept()
    eta = np.full(K, -1.0 if model == D.LR else -2.0)
    pool = rng.choice(K, size=4_000, replace=False)         # rows the sparse columns share
    for c in range(n_sparse):
        n = int(rng.integers(5, 400))
        rows = rng.choice(pool, size=n, replace=False)
        vals = rng.normal(0.0, 1.0, size=n)
        b.sparse(rows, vals)
        if c % 3 == 0:
            eta[rows] += 0.5 * vals
    counts = np.maximum(1, (K * 0.5 * np.arange(1, n_ind + 1) ** -0.9)).astype(int)
    for c in range(n_ind):
        rows = rng.choice(K, size=min(K, counts[c]), replace=False)
        b.indicator(rows)
        if c % 4 == 0:
            eta[rows] += rng.normal(0.0, 0.5)
    if model == D.LR:
        y = (rng.random(K) < 1.0 / (1.0 + np.exp(-eta))).astype(float)
    else:
        y = rng.poisson(np.exp(np.minimum(eta, 5.0))).astype(float)
    return b.build(model, y, has_intercept=True)


def _oracle_fit(data, variance, weights, tol):
    from oracle import oracle as O
    return O.port().fit(data, D.PRIOR_LAPLACE, variance,
                        control=O.make_control(tolerance=tol, convergence_type=D.CONV_GRADIENT), exclude=[0],
                        weights=weights)


@pytest.fixture
def cluster_size():
    old = os.environ.get("CYC_BATCH_CLUSTER")
    yield lambda c: os.environ.__setitem__("CYC_BATCH_CLUSTER", str(c))
    if old is None:
        os.environ.pop("CYC_BATCH_CLUSTER", None)
    else:
        os.environ["CYC_BATCH_CLUSTER"] = old


@pytest.mark.parametrize("model", [D.LR, D.PR])
@pytest.mark.parametrize("clusters", [1, 3, 8])
def test_cv_grid_matches_oracle(cuda_lib, cluster_size, model, clusters):
    """FP64 state at tolerance 1e-7 (gradient rule): every fit is the
    oracle's under the precision contract, cycle for cycle, and its held-out
    predictive log likelihood is the oracle's for its coefficients."""
    from cyclops_b200 import api
    from oracle import oracle as O
    cluster_size(clusters)
    data = _mixed_data(model)
    n_folds = 5
    masks = api.cv_fold_weights(data.K, n_folds, 31)
    folds = api.fold_ids_from_weights(masks)
    variances = [D.laplace_variance(lam) for lam in (1.0, 10.0)]
    tol = 1e-7
    prior = api.PriorSpec(D.PRIOR_LAPLACE, 1.0, [0])
    res = api.cv_grid_fit(data, prior, folds, n_folds, variances, api.create_control(tolerance=tol))
    lib = O.port()
    for i, fit in enumerate(res.fits):
        v, f = variances[i // n_folds], i % n_folds
        ref = _oracle_fit(data, v, masks[f], tol)
        assert ref.return_flag == 0
        assert_contract(fit, ref, what=i)
        held = (masks[f] == 0).astype(float)
        pll = lib.predictive_loglik(data, fit.beta, held)
        assert rel_err(res.pred_loglik[i], pll) < 1e-9, (i, res.pred_loglik[i], pll)
    for v in range(len(variances)):
        assert rel_err(res.grid_mean[v], np.mean(res.pred_loglik[v * n_folds:(v + 1) * n_folds])) < 1e-12


@pytest.mark.parametrize("model", [D.LR, D.PR])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("clusters", [1, 3, 8])
def test_cv_grid_tight_contract(cuda_lib, cluster_size, model, precision, clusters):
    """Both sides converged tightly (Mittal rule, tolerance 1e-12): beta 1e-6
    relative (1e-9 absolute), log likelihood 1e-9 relative, for FP64 state
    and for FP32 state with compensated sums followed by the FP64 polish,
    at 1, 3 and 8 CTAs.  Cycle counts are not compared here: a relative
    log-likelihood change of 1e-12 is at the rounding level of the
    likelihood's sum over 20k rows (the two sides' sums differ by ~5e-13
    relative), so where exactly the stopping test fires is rounding, not
    arithmetic; the cycle-for-cycle check is test_cv_grid_matches_oracle's."""
    from cyclops_b200 import api
    from oracle import oracle as O
    cluster_size(clusters)
    data = _mixed_data(model, K=20_000, n_sparse=60, n_ind=150, seed=7)
    n_folds = 4
    masks = api.cv_fold_weights(data.K, n_folds, 13)
    folds = api.fold_ids_from_weights(masks)
    variances = [D.laplace_variance(lam) for lam in (2.0, 20.0)]
    prior = api.PriorSpec(D.PRIOR_LAPLACE, 1.0, [0])
    ctl = api.create_control(tolerance=1e-12, convergence_type="mittal", precision=precision,
                             polish_tolerance=1e-5, max_iterations=5000)
    res = api.cv_grid_fit(data, prior, folds, n_folds, variances, ctl)
    octl = O.make_control(tolerance=1e-12, convergence_type=D.CONV_MITTAL, max_iterations=5000)
    for i, fit in enumerate(res.fits):
        v, f = variances[i // n_folds], i % n_folds
        ref = O.port().fit(data, D.PRIOR_LAPLACE, v, control=octl, exclude=[0], weights=masks[f])
        assert_contract(fit, ref, iterations=False, what=i)


def test_cluster_sizes_agree(cuda_lib, cluster_size):
    """The same grid split over 1, 2, 5 and 8 CTAs: only the order of the
    cross-CTA sums differs, so the fits agree far inside the tolerance."""
    from cyclops_b200 import api
    data = _mixed_data(D.LR, seed=9)
    masks = api.cv_fold_weights(data.K, 4, 3)
    folds = api.fold_ids_from_weights(masks)
    prior = api.PriorSpec(D.PRIOR_LAPLACE, 1.0, [0])
    ctl = api.create_control(tolerance=1e-8)
    variances = [D.laplace_variance(10.0)] * 2
    out = {}
    for c in (1, 2, 5, 8):
        cluster_size(c)
        out[c] = np.array([f.beta for f in api.cv_grid_fit(data, prior, folds, 4, variances, ctl).fits])
    for c in (2, 5, 8):
        assert np.max(np.abs(out[c] - out[1]) / np.maximum(np.abs(out[1]), 1.0)) < 1e-6, c


@pytest.mark.parametrize("name", ["lr_normal_weighted", "lr_laplace_small", "cpr_normal", "clr_normal_weighted"])
def test_weighted_cv_grid_matches_oracle(cuda_lib, name):
    """Observation weights in CV (CrossValidationSelector with the fit's
    weights): each fold trains at the weights outside it and is scored at
    the weights inside it; fits and held-out log likelihoods against the
    restatement oracle run on the same masks."""
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden(name)
    base = np.ones(data.K) if s["weights"] is None else np.asarray(s["weights"], float)
    w = base * (1.0 + (np.arange(data.K) % 3))                              # non-0/1 weights
    n_folds = 5
    fold = (np.arange(data.K) * 7 % n_folds).astype(np.int32)
    variances = [float(s["variance"]), 2.0 * float(s["variance"])]
    prior = api.PriorSpec(int(s["prior"]), 1.0, exclude_for(data))
    ctl = api.create_control()
    res = api.cv_grid_fit(data, prior, fold, n_folds, variances, ctl, weights=w)
    octl = O.make_control()
    for i, fit in enumerate(res.fits):
        v, f = variances[i // n_folds], i % n_folds
        train = np.where(fold == f, 0.0, w)
        held = np.where(fold == f, w, 0.0)
        ref = O.port().fit(data, int(s["prior"]), v, control=octl, weights=train)
        if ref.return_flag != 0:                     # not converged: NaN, as the reference's driver records
            assert fit.return_flag == ref.return_flag and fit.iterations == ref.iterations
            assert np.isnan(res.pred_loglik[i])
            continue
        assert_contract(fit, ref, what=i)
        want = O.port().predictive_loglik(data, ref.beta, held, weights=train)
        assert abs(res.pred_loglik[i] - want) <= 1e-8 * abs(want), (i, res.pred_loglik[i], want)


@pytest.mark.parametrize("name,weighted", [("cox_laplace", False), ("cox_strata", False), ("cox_ties_weighted", True)])
def test_cox_cv_grid_matches_oracle(cuda_lib, name, weighted):
    """Cox cross-validation grids (folds by row, R's choice for these
    shapes): every fold's fit is the oracle's on its training weights, and
    its held-out predictive log likelihood is the oracle's, scored against
    the training rows' risk sets."""
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden(name)
    n_folds = 5
    masks = api.cv_fold_weights(data.K, n_folds, 23)
    folds = api.fold_ids_from_weights(masks)
    w = np.asarray(s["weights"], float) * (1.0 + (np.arange(data.K) % 2)) if weighted else None
    variances = [float(s["variance"]), 4.0 * float(s["variance"])]
    prior = api.PriorSpec(int(s["prior"]), 1.0, exclude_for(data))
    res = api.cv_grid_fit(data, prior, folds, n_folds, variances, api.create_control(), weights=w)
    base = np.ones(data.K) if w is None else w
    for i, fit in enumerate(res.fits):
        v, f = variances[i // n_folds], i % n_folds
        train = masks[f] * base
        held = (1.0 - masks[f]) * base
        ref = O.port().fit(data, int(s["prior"]), v, control=O.make_control(), weights=train)
        assert ref.return_flag == 0
        assert_contract(fit, ref, what=(name, i))
        want = O.port().predictive_loglik(data, ref.beta, held, weights=train)
        assert abs(res.pred_loglik[i] - want) <= 1e-8 * abs(want), (i, res.pred_loglik[i], want)
    for v in range(len(variances)):
        assert rel_err(res.grid_mean[v], np.mean(res.pred_loglik[v * n_folds:(v + 1) * n_folds])) < 1e-12

"""Batched device-resident CCD (cyc_batch_fit): every fit of a batch equals
the reference engine's fit of the same (weights, prior) on its own, under
the precision contract (same cycles, beta 1e-6 relative, log likelihood
1e-9 relative), at the default tolerance as well as converged tightly."""
import numpy as np
import pytest

from conftest import assert_contract, exclude_for, load_golden
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu


def _ref_fit(data, prior, variance, weights, tol=1e-6, conv=D.CONV_GRADIENT, max_iterations=1000):
    from oracle import oracle as O
    ctl = O.make_control(tolerance=tol, convergence_type=conv, max_iterations=max_iterations)
    return O.port().fit(data, prior, variance, control=ctl, weights=weights)


@pytest.mark.parametrize("name", ["lr_laplace_small", "lr_normal_weighted", "pr_laplace_weighted",
                                  "clr_laplace", "clr_normal_weighted", "cpr_normal", "pr_offset_normal"])
@pytest.mark.parametrize("nfits", [1, 6, 11])
def test_batch_fits_match_reference(cuda_lib, name, nfits):
    from cyclops_b200 import api
    data, s = load_golden(name)
    rng = np.random.default_rng(nfits)
    var0 = float(s["variance"])
    variances = [var0 * (1.0 + 0.5 * (f % 3)) for f in range(nfits)]
    weights = []
    for f in range(nfits):
        if f == 0:
            weights.append(s["weights"])
        elif data.model in (D.CLR, D.CPR):
            strata = data.strata()
            keep = (rng.random(strata.max() + 1) > 0.2).astype(float)
            weights.append(keep[strata])
        else:
            weights.append((rng.random(data.K) > 0.2).astype(float))
    prior = api.PriorSpec(int(s["prior"]), var0, exclude_for(data))
    fits = api.batch_fit(data, prior, variances, weights, api.create_control(tolerance=1e-6))
    for f in range(nfits):
        ref = _ref_fit(data, int(s["prior"]), variances[f], weights[f])
        assert_contract(fits[f], ref, what=(name, f))


@pytest.mark.parametrize("name", ["lr_c1", "clr_laplace", "pr_laplace_weighted"])
def test_mixed_precision_batch_reaches_fp64_fit(cuda_lib, name):
    """FP32 state with compensated sums, then the FP64 polish: the result is
    the FP64 oracle's fit to 1e-6 relative when both are converged tightly."""
    from cyclops_b200 import api
    data, s = load_golden(name)
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    ctl = api.create_control(tolerance=1e-12, convergence_type="mittal", precision="mixed", polish_tolerance=1e-5,
                             max_iterations=3000)
    fits = api.batch_fit(data, prior, [float(s["variance"])] * 3, [s["weights"]] * 3, ctl)
    ref = _ref_fit(data, int(s["prior"]), float(s["variance"]), s["weights"], tol=1e-12, conv=D.CONV_MITTAL,
                   max_iterations=3000)
    for fit in fits:
        # the reported cycles of a mixed fit are its FP64 phase's
        assert_contract(fit, ref, iterations=False, what=name)


@pytest.mark.parametrize("name", ["lr_c1", "lr_normal_weighted", "pr_offset_normal", "clr_laplace", "cpr_normal"])
def test_fp64_batch_tight_contract(cuda_lib, name):
    """FP64 batch, Mittal 1e-12 on both sides: the fits are the oracle's
    cycle for cycle."""
    from cyclops_b200 import api
    data, s = load_golden(name)
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    ctl = api.create_control(tolerance=1e-12, convergence_type="mittal", max_iterations=5000)
    variances = [float(s["variance"]), 2.0 * float(s["variance"])]
    fits = api.batch_fit(data, prior, variances, [s["weights"]] * 2, ctl)
    for v, fit in zip(variances, fits):
        ref = _ref_fit(data, int(s["prior"]), v, s["weights"], tol=1e-12, conv=D.CONV_MITTAL, max_iterations=5000)
        assert_contract(fit, ref, what=(name, v))


def test_cv_folds_times_grid(cuda_lib):
    """5 folds x 3 prior variances from the reference's fold rule, as one batch."""
    from cyclops_b200 import api
    data, s = load_golden("lr_laplace_small")
    folds = api.cv_fold_weights(data.K, 5, 17)
    lams = [0.5, 1.0, 2.0]
    variances, weights = [], []
    for lam in lams:
        for f in range(5):
            variances.append(D.laplace_variance(lam))
            weights.append(folds[f])
    prior = api.PriorSpec(D.PRIOR_LAPLACE, 1.0, exclude_for(data))
    fits = api.batch_fit(data, prior, variances, weights, api.create_control())
    for i, fit in enumerate(fits):
        ref = _ref_fit(data, D.PRIOR_LAPLACE, variances[i], weights[i])
        assert_contract(fit, ref, what=i)


@pytest.mark.parametrize("name", ["cox_laplace", "cox_strata", "cox_ties_weighted"])
@pytest.mark.parametrize("nfits", [1, 6, 11])
def test_cox_batch_fits_match_reference(cuda_lib, name, nfits):
    """Cox fits of a batch (each with the risk sets of its own weights) run
    as concurrent single-fit solves: every fit is the oracle's at its
    weights and variance, under the precision contract."""
    from cyclops_b200 import api
    data, s = load_golden(name)
    rng = np.random.default_rng(100 + nfits)
    var0 = float(s["variance"])
    base = np.ones(data.K) if s["weights"] is None else np.asarray(s["weights"], float)
    variances = [var0 * (1.0 + 0.5 * (f % 3)) for f in range(nfits)]
    weights = [s["weights"] if f == 0 else base * (rng.random(data.K) > 0.2) for f in range(nfits)]
    prior = api.PriorSpec(int(s["prior"]), var0, exclude_for(data))
    fits = api.batch_fit(data, prior, variances, weights, api.create_control())
    st = api.last_run_stats()
    assert st["cycles"] == sum(f.iterations for f in fits) and st["launches"] > 0
    for f in range(nfits):
        ref = _ref_fit(data, int(s["prior"]), variances[f], weights[f])
        assert_contract(fits[f], ref, what=(name, f))


def test_cox_bootstrap_replicates(cuda_lib):
    """Bootstrap replicates of a stratified Cox fit (BootstrapSelector's
    per-row draws) as one cyc_batch_fit call."""
    from cyclops_b200 import api
    data, s = load_golden("cox_strata")
    W = api.bootstrap_weights(data.K, 5, 7)
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    fits = api.batch_fit(data, prior, [float(s["variance"])] * 5, list(W), api.create_control())
    for r, fit in enumerate(fits):
        assert_contract(fit, _ref_fit(data, int(s["prior"]), float(s["variance"]), W[r]), what=r)


def test_concurrent_fit_count_does_not_change_fits(cuda_lib, monkeypatch):
    """One, three or eight Cox fits in flight at a time: each fit is its own
    single-fit solve, so the results are bitwise the same."""
    from cyclops_b200 import api
    data, s = load_golden("cox_strata")
    rng = np.random.default_rng(3)
    weights = [(rng.random(data.K) > 0.25).astype(float) for _ in range(9)]
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    got = {}
    for slots in (1, 3, 8):
        monkeypatch.setenv("CYC_CONCURRENT_FITS", str(slots))
        got[slots] = api.batch_fit(data, prior, [float(s["variance"])] * 9, weights, api.create_control())
    for slots in (3, 8):
        for a, b in zip(got[1], got[slots]):
            assert np.array_equal(a.beta, b.beta) and a.iterations == b.iterations
            assert a.log_likelihood == b.log_likelihood


@pytest.mark.parametrize("name", ["lr_laplace_small", "clr_laplace", "pr_laplace_weighted"])
def test_bootstrap_replicates_as_one_batch(cuda_lib, name):
    """Bootstrap replicates (BootstrapSelector's weights: per row, or per
    matched stratum for clr) fitted as one batched solve; each replicate is
    the oracle's fit at its weights (a cold start, as every fit of a batch)."""
    from cyclops_b200 import api
    data, s = load_golden(name)
    ids = data.strata() if data.model in (D.CLR, D.CPR) else None
    W = api.bootstrap_weights(data.K, 6, 42, ids=ids)
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    fits = api.batch_fit(data, prior, [float(s["variance"])] * 6, list(W), api.create_control())
    for r, fit in enumerate(fits):
        ref = _ref_fit(data, int(s["prior"]), float(s["variance"]), W[r])
        assert_contract(fit, ref, what=(name, r))

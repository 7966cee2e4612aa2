"""Generates tests/golden/*.npz from the reference Cyclops engine.

Each fixture holds a small seeded problem (the arrays themselves, so the
fixture does not depend on the generator) and what the reference engine,
compiled from its own sources (oracle/_ref/libcyclops_ref.so), returns for
it: the fitted coefficients, log likelihood, log prior, iteration count and
return flag of CyclicCoordinateDescent::update, the per-column
(gradient, Hessian) of the engine at a fixed coefficient vector, and the
linear predictor there.  The CV fold masks come from the reference's
CrossValidationSelector.

    python tests/golden/make_golden.py      # needs the reference sources
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from cyclops_b200 import data as D  # noqa: E402
from oracle import oracle as O      # noqa: E402


def cases():
    lam01 = D.laplace_variance(0.1)
    c = {}
    # the reference's CPU-runnable configuration: 10k x 1k indicators at 1 %,
    # Laplace lambda = 0.1 (variance 200), default control
    c["lr_c1"] = dict(data=D.synth_logistic(seed=1), prior=D.PRIOR_LAPLACE, variance=lam01)
    c["lr_laplace_small"] = dict(data=D.synth_logistic(K=3000, P=200, density=0.02, n_true=20, seed=21),
                                 prior=D.PRIOR_LAPLACE, variance=D.laplace_variance(1.0))
    rng = np.random.default_rng(5)
    d = D.synth_logistic(K=3000, P=150, density=0.02, n_true=20, seed=22)
    c["lr_normal_weighted"] = dict(data=d, prior=D.PRIOR_NORMAL, variance=0.5,
                                   weights=(rng.random(d.K) > 0.25).astype(float))
    c["lr_lange"] = dict(data=D.synth_logistic(K=2000, P=80, density=0.03, n_true=10, seed=23),
                         prior=D.PRIOR_NORMAL, variance=2.0, convergence=D.CONV_LANGE, tolerance=1e-8)
    c["lr_zhang_oles"] = dict(data=D.synth_logistic(K=2000, P=80, density=0.03, n_true=10, seed=24),
                              prior=D.PRIOR_LAPLACE, variance=D.laplace_variance(2.0),
                              convergence=D.CONV_ZHANG_OLES, tolerance=1e-7)
    c["lr_flat"] = dict(data=D.synth_logistic(K=4000, P=12, density=0.2, n_true=6, seed=25),
                        prior=D.PRIOR_NONE, variance=1.0, convergence=D.CONV_MITTAL, tolerance=1e-10)
    c["pr_offset_normal"] = dict(data=D.synth_poisson(K=4000, P=200, per_row=6, n_dense=3, n_true=25, seed=31),
                                 prior=D.PRIOR_NORMAL, variance=1.0)
    d = D.synth_poisson(K=3000, P=120, per_row=5, n_dense=2, n_true=15, seed=32, offset=False)
    c["pr_laplace_weighted"] = dict(data=d, prior=D.PRIOR_LAPLACE, variance=D.laplace_variance(0.5),
                                    weights=(rng.random(d.K) > 0.3).astype(float))
    c["clr_laplace"] = dict(data=D.synth_conditional(K=4000, P=150, density=0.02, seed=41),
                            prior=D.PRIOR_LAPLACE, variance=D.laplace_variance(1.0))
    d = D.synth_conditional(K=3000, P=100, density=0.03, seed=42)
    c["clr_normal_weighted"] = dict(data=d, prior=D.PRIOR_NORMAL, variance=1.0,
                                    weights=np.repeat((rng.random(d.K // 5) > 0.2).astype(float), 5))
    c["cpr_normal"] = dict(data=D.synth_conditional(K=3000, P=100, density=0.03, seed=43, model=D.CPR),
                           prior=D.PRIOR_NORMAL, variance=1.0)
    c["cox_laplace"] = dict(data=D.synth_cox(K=3000, P=120, density=0.02, n_true=30, seed=51),
                            prior=D.PRIOR_LAPLACE, variance=D.laplace_variance(2.0))
    c["cox_strata"] = dict(data=D.synth_cox(K=3000, P=120, density=0.02, n_strata=25, n_true=30, seed=52),
                           prior=D.PRIOR_LAPLACE, variance=D.laplace_variance(2.0))
    d = D.synth_cox(K=3000, P=100, density=0.02, n_strata=4, n_true=30, seed=53, ties=1)
    c["cox_ties_weighted"] = dict(data=d, prior=D.PRIOR_NORMAL, variance=1.0,
                                  weights=(rng.random(d.K) > 0.2).astype(float))
    c["cox_indicator"] = dict(data=D.synth_cox(K=3000, P=100, density=0.03, n_true=30, seed=54, indicator=True),
                              prior=D.PRIOR_NORMAL, variance=1.0)
    # edge: an empty indicator column and a dense column under Laplace
    d = D.synth_logistic(K=1500, P=40, density=0.05, n_true=5, seed=61)
    b = D.ColumnBuilder(d.K).intercept()
    b.dense(np.random.default_rng(7).normal(size=d.K))
    for j in range(1, d.J):
        rows, _ = d.column(j)
        b.indicator(rows if j != 5 else [])
    c["lr_empty_column"] = dict(data=b.build(D.LR, d.y, has_intercept=True), prior=D.PRIOR_LAPLACE,
                                variance=D.laplace_variance(0.5))
    return c


def save_case(name, spec):
    d: D.CyclopsData = spec["data"]
    ctl = O.make_control(tolerance=spec.get("tolerance", 1e-6),
                         convergence_type=spec.get("convergence", D.CONV_GRADIENT),
                         use_kkt_swindle=spec.get("swindle", 0))
    w = spec.get("weights")
    fit = O.ref().fit(d, spec["prior"], spec["variance"], control=ctl, weights=w)
    rng = np.random.default_rng(99)
    beta_probe = fit.beta + np.where(fit.beta != 0, 0.05 * rng.normal(size=d.J), 0.0)
    if d.has_offset:
        beta_probe[0] = 1.0
    g, h, xb, ll = O.ref().probe(d, beta_probe, spec["prior"], spec["variance"], weights=w)
    arrays = dict(
        model=d.model, y=d.y, col_format=d.col_format, col_ptr=d.col_ptr, col_idx=d.col_idx,
        val_ptr=d.val_ptr, col_val=d.col_val,
        pid=d.pid if d.pid is not None else np.zeros(0, np.int32),
        time=d.time if d.time is not None else np.zeros(0),
        has_offset=int(d.has_offset), has_intercept=int(d.has_intercept),
        prior=spec["prior"], variance=spec["variance"],
        weights=w if w is not None else np.zeros(0),
        tolerance=ctl.tolerance, convergence=ctl.convergence_type,
        beta=fit.beta, log_likelihood=fit.log_likelihood, log_prior=fit.log_prior,
        iterations=fit.iterations, return_flag=fit.return_flag,
        probe_beta=beta_probe, probe_gradient=g, probe_hessian=h, probe_xbeta=xb, probe_loglik=ll,
    )
    if spec.get("swindle"):
        arrays["swindle"] = 1
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(f"{name:22s} K={d.K:6d} J={d.J:5d} nnz={d.nnz:7d} it={fit.iterations:4d} "
          f"flag={fit.return_flag} ll={fit.log_likelihood:.8f}")


def save_cv():
    K = 1003
    ids = np.arange(K, dtype=np.int32)
    by_row = O.ref_cv_weights(K, ids, 10, 123, by_row=True, n_reps=2)
    pid = np.repeat(np.arange(201, dtype=np.int32), 5)[:K]
    by_pid = O.ref_cv_weights(K, pid, 5, 77, by_row=False, n_reps=1)
    np.savez_compressed(os.path.join(HERE, "cv_folds.npz"), K=K, by_row=by_row, pid=pid, by_pid=by_pid,
                        seed_row=123, seed_pid=77)
    print("cv_folds", by_row.shape, by_pid.shape)


def save_bootstrap():
    """BootstrapSelector's replicate weights (by unit id), per row and with
    matched strata of 5 rows as the units."""
    K = 1003
    ids = np.arange(K, dtype=np.int32)
    by_row = O.ref_bootstrap_weights(K, ids, 8, 123)
    pid = np.repeat(np.arange(201, dtype=np.int32), 5)[:K]
    by_pid = O.ref_bootstrap_weights(K, pid, 4, 77)
    np.savez_compressed(os.path.join(HERE, "bootstrap_weights.npz"), K=K, by_row=by_row, pid=pid, by_pid=by_pid,
                        seed_row=123, seed_pid=77)
    print("bootstrap_weights", by_row.shape, by_pid.shape)


def ingest_tables(model_type, seed, with_values=True, n=80, m=400):
    """Unsorted long-format tables with the awkward cases: rowIds in random
    order, covariate rows without an outcome, zero values, columns that start
    as indicators and hold a non-0/1 value later, ties in Cox times."""
    rng = np.random.default_rng(seed)
    outcomes = {"rowId": rng.permutation(np.arange(1000, 1000 + n)).astype(np.int64),
                "y": rng.integers(0, 2, n).astype(np.float64),
                "stratumId": rng.integers(0, max(2, n // 5), n).astype(np.int64),
                "time": rng.choice([0.25, 0.5, 1.0, 2.0, 3.0], n).astype(np.float64)}
    rows = rng.integers(990, 1000 + n, m).astype(np.int64)
    cids = rng.integers(1, 15, m).astype(np.int64)
    key = rows * 100 + cids
    _, u = np.unique(key, return_index=True)
    u = rng.permutation(u)
    cov = {"rowId": rows[u], "covariateId": cids[u]}
    if with_values:
        cov["covariateValue"] = rng.choice([0.0, 1.0, 1.0, 1.0, 2.5, -0.75], u.size).astype(np.float64)
    return outcomes, cov


def save_ingest():
    """The reference loader's result for each model type (tables sorted by
    the R layer's rules, then ModelData::loadY / loadX / loadMultipleX)."""
    from cyclops_b200 import ingest
    for mt, seed, vals in [("lr", 1, True), ("pr", 2, True), ("clr", 3, True), ("cox", 4, True), ("lr", 5, False)]:
        model = ingest._MODELS[mt]
        outcomes, cov = ingest_tables(mt, seed, vals)
        outs = ingest.sort_outcomes(model, outcomes)
        covs = ingest.sort_covariates(model, cov, outs)
        ref = O.ref_ingest(model, {k: outs[k] for k in ("rowId", "y", "stratumId", "time") if outs[k] is not None},
                           {"rowId": covs["rowId"], "covariateId": covs["covariateId"],
                            "covariateValue": covs["covariateValue"]},
                           mt in ("lr", "pr"), mt in ("pr", "cpr"))
        name = f"ingest_{mt}_{seed}"
        arrays = {"model_type": mt, **{"in_" + k: v for k, v in outcomes.items()},
                  **{"cov_" + k: v for k, v in cov.items()},
                  **{"ref_" + k: v for k, v in ref.items() if v is not None}}
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, "J", len(ref["col_format"]), "nnz", int(ref["col_ptr"][-1]))


SWINDLE_CASES = ["lr_c1", "lr_laplace_small", "lr_zhang_oles", "lr_empty_column", "pr_laplace_weighted",
                 "clr_laplace", "cox_laplace", "cox_strata"]


def save_swindle():
    """The Laplace problems fitted with the KKT swindle (ModeFindingArguments
    useKktSwindle, CyclicCoordinateDescent::kktSwindle,
    src/cyclops/CyclicCoordinateDescent.cpp:636-814): swindle_<case>.npz."""
    all_cases = cases()
    for name in SWINDLE_CASES:
        save_case("swindle_" + name, dict(all_cases[name], swindle=1))


# (fixture, columns, override_no_regularization, include_penalty, KKT swindle)
PROFILE_CASES = [("lr_flat", [0, 1, 2, 3], False, True, 0),
                 ("lr_normal_weighted", [0, 3, 7], True, True, 0),
                 ("clr_normal_weighted", [0, 5, 9], True, False, 0),
                 ("pr_offset_normal", [1, 2, 8], True, True, 0),
                 ("cox_ties_weighted", [0, 4], True, True, 0),
                 ("lr_laplace_small", [0, 1, 2], True, True, 1)]


def save_profile():
    """Profile-likelihood bounds (CcdInterface::profileModel with one thread,
    src/cyclops/CcdInterface.cpp:262-420) at the 95 % threshold
    qchisq(0.95, 1) / 2, and the profile log likelihood at 9 points around
    the estimate of the last column (evaluateProfileModel, :527-618):
    profile_<case>.npz holds the problem, the columns, the reference's lower /
    upper bounds and refit counts, the points and their values."""
    all_cases = cases()
    threshold = 1.920729410347062          # qchisq(0.95, df = 1) / 2
    for name, cols, override, penalty, swindle in PROFILE_CASES:
        spec = all_cases[name]
        d = spec["data"]
        ctl = O.make_control(tolerance=spec.get("tolerance", 1e-6),
                             convergence_type=spec.get("convergence", D.CONV_GRADIENT), use_kkt_swindle=swindle)
        w = spec.get("weights")
        lo, up, ev, fit = O.ref().profile(d, cols, spec["prior"], spec["variance"], threshold, penalty, override,
                                          control=ctl, weights=w)
        # getCyclopsProfileLogLikelihood (evaluateProfileModel) on the last column
        points = fit.beta[cols[-1]] + np.linspace(-0.6, 0.6, 9)
        values = O.ref().profile_points(d, cols[-1], points, spec["prior"], spec["variance"], penalty,
                                        control=ctl, weights=w)
        arrays = dict(
            model=d.model, y=d.y, col_format=d.col_format, col_ptr=d.col_ptr, col_idx=d.col_idx,
            val_ptr=d.val_ptr, col_val=d.col_val,
            pid=d.pid if d.pid is not None else np.zeros(0, np.int32),
            time=d.time if d.time is not None else np.zeros(0),
            has_offset=int(d.has_offset), has_intercept=int(d.has_intercept),
            prior=spec["prior"], variance=spec["variance"],
            weights=w if w is not None else np.zeros(0),
            tolerance=ctl.tolerance, convergence=ctl.convergence_type, swindle=swindle,
            columns=np.asarray(cols, np.int32), threshold=threshold, include_penalty=int(penalty),
            override=int(override), lower=lo, upper=up, evaluations=ev, beta=fit.beta,
            point_column=int(cols[-1]), points=points, point_values=values,
        )
        np.savez_compressed(os.path.join(HERE, "profile_" + name + ".npz"), **arrays)
        print(f"profile_{name:20s} cols={cols} evals={ev.tolist()}")


REF_TESTS = os.path.join(os.environ.get("CYCLOPS_REFERENCE", "/root/reference"), "tests", "testthat")


def _r_vector(text, name):
    """The numbers of `name <- c(...)` or `name = c(...)` (first occurrence)."""
    m = re.search(name + r"\s*(?:<-|=)\s*c\(([^)]*)\)", text)
    if not m:
        raise RuntimeError(f"{name} not found in the reference test")
    return np.array([float(v) for v in m.group(1).split(",")])


def _r_gl(text, name):
    """R's gl(n, k, length) factor levels (1-based) for `name = gl(...)`."""
    m = re.search(name + r"\s*(?:<-|=)\s*gl\((\d+)\s*,\s*(\d+)(?:\s*,\s*(\d+))?\)", text)
    n, k = int(m.group(1)), int(m.group(2))
    length = int(m.group(3)) if m.group(3) else n * k
    return np.resize(np.repeat(np.arange(1, n + 1), k), length)


def _r_tables(text):
    """Every read.table(..., text = "...") block: header + numeric rows."""
    out = []
    for block in re.findall(r'text\s*=\s*"([^"]*)"', text):
        lines = [l.strip() for l in block.strip().splitlines() if l.strip()]
        cols = [c.strip() for c in lines[0].split(",")]
        rows = np.array([[float(v) for v in l.split(",")] for l in lines[1:]])
        out.append({c: rows[:, i] for i, c in enumerate(cols)})
    return out


def small_designs():
    """The tiny designs of the reference's own tests, read from its test files
    (tests/testthat/test-smallCox.R, test-smallBernoulli.R,
    test-smallPoisson.R) and its text fixture inst/extdata/infert_ccd.txt, in
    the formats those tests use."""
    from cyclops_b200 import ingest
    out = {}
    cox = _r_tables(open(os.path.join(REF_TESTS, "test-smallCox.R")).read())

    def cox_data(t, strata, weights=None, x1=None):
        n = len(t["length"])
        rid = np.arange(1, n + 1, dtype=np.int64)
        outcomes = {"rowId": rid, "y": t["event"], "time": t["length"],
                    "stratumId": (t["x2"] if strata else np.zeros(n)).astype(np.int64)}
        if weights is not None:
            outcomes["weights"] = weights
        x1v = t["x1"] if x1 is None else x1
        cid = [np.full(n, 1)] + ([] if strata else [np.full(n, 2)])
        vals = [x1v] + ([] if strata else [t["x2"]])
        cov = {"rowId": np.concatenate([rid] * len(cid)), "covariateId": np.concatenate(cid).astype(np.int64),
               "covariateValue": np.concatenate(vals)}
        return ingest.convert_to_cyclops_data(outcomes, cov, model_type="cox")

    out["small_cox_noties"] = cox_data(cox[0], False)
    out["small_cox_noties_strata"] = cox_data(cox[0], True)
    out["small_cox_timeties"] = cox_data(cox[1], False)
    out["small_cox_failties"] = cox_data(cox[2], False)
    out["small_cox_failties_risk"] = cox_data(cox[3], False)
    out["small_cox_failties_strata"] = cox_data(cox[3], True)
    # each row twice, the first copy weighted 0 and two of those given other
    # x1 values: the fit equals small_cox_failties_strata (zero weight = removal)
    t = {k: np.repeat(v, 2) for k, v in cox[3].items()}
    x1 = t["x1"].copy()
    x1[0], x1[4] = 5.0, 6.0
    out["small_cox_zero_weights"] = cox_data(t, True, weights=np.tile([0.0, 1.0], len(cox[3]["x1"])), x1=x1)

    bern = open(os.path.join(REF_TESTS, "test-smallBernoulli.R")).read()
    bid, nn, yy = (_r_vector(bern, v) for v in ("binomial_bid", "binomial_n", "binomial_y"))
    log_bid = np.log(np.concatenate([np.repeat(bid, (nn - yy).astype(int)), np.repeat(bid, yy.astype(int))]))
    y = np.concatenate([np.zeros(int(np.sum(nn - yy))), np.ones(int(np.sum(yy)))])
    K = y.size
    out["small_lr_dense"] = (D.ColumnBuilder(K).intercept().dense(log_bid).build(D.LR, y, has_intercept=True), None)
    nz = np.flatnonzero(log_bid != 0)
    out["small_lr_sparse"] = (D.ColumnBuilder(K).intercept().sparse(nz, log_bid[nz])
                              .build(D.LR, y, has_intercept=True), None)

    # the reference's CCD text fixture of the infert matched case-control
    # data (inst/extdata/infert_ccd.txt: stratum, case, covariate:value ...),
    # conditional logistic as test-smallCLR.R fits it
    rows, cids, vals, strata, ys = [], [], [], [], []
    path = os.path.join(os.path.dirname(os.path.dirname(REF_TESTS)), "inst", "extdata", "infert_ccd.txt")
    for i, line in enumerate(l for l in open(path) if l.strip() and not l.startswith("#")):
        f = line.split()
        strata.append(int(f[0]))
        ys.append(float(f[1]))
        for item in f[2:]:
            c, v = item.split(":")
            rows.append(i + 1)
            cids.append(int(c))
            vals.append(float(v))
    n = len(ys)
    out["small_clr_infert"] = ingest.convert_to_cyclops_data(
        {"rowId": np.arange(1, n + 1, dtype=np.int64), "y": np.asarray(ys), "stratumId": np.asarray(strata, np.int64)},
        {"rowId": np.asarray(rows, np.int64), "covariateId": np.asarray(cids, np.int64),
         "covariateValue": np.asarray(vals)}, model_type="clr")

    pois = open(os.path.join(REF_TESTS, "test-smallPoisson.R")).read()
    counts = _r_vector(pois, "counts")
    outcome, treatment = _r_gl(pois, "outcome"), _r_gl(pois, "treatment")
    K = counts.size
    dummies = [(outcome == 2), (outcome == 3), (treatment == 2), (treatment == 3)]
    b = D.ColumnBuilder(K).intercept()
    for dmy in dummies:
        b.dense(dmy.astype(float))
    out["small_pr_dense"] = (b.build(D.PR, counts, has_intercept=True), None)
    b = D.ColumnBuilder(K).intercept().dense(dummies[0].astype(float)).dense(dummies[1].astype(float))
    for dmy in dummies[2:]:
        b.indicator(np.flatnonzero(dmy))
    out["small_pr_indicator"] = (b.build(D.PR, counts, has_intercept=True), None)
    return out


def save_small():
    """small_<design>.npz: a design from the reference's own tests, the
    reference engine's unpenalised fit of it at the default control and at a
    tight one (Mittal 1e-17: until the log likelihood stops changing in
    double precision), and an independent Newton-Raphson MLE
    (oracle/newton.py) of the same likelihood."""
    from oracle import newton
    for name, (d, w) in small_designs().items():
        ex = [1 if d.has_offset else 0] if d.has_intercept else []
        fit = O.ref().fit(d, D.PRIOR_NONE, 1.0, control=O.make_control(), exclude=ex, weights=w)
        tight = O.ref().fit(d, D.PRIOR_NONE, 1.0, exclude=ex, weights=w,
                            control=O.make_control(tolerance=1e-17, convergence_type=D.CONV_MITTAL,
                                                   max_iterations=100000))
        nb, nll = newton.newton_fit(d, w)
        arrays = dict(
            model=d.model, y=d.y, col_format=d.col_format, col_ptr=d.col_ptr, col_idx=d.col_idx,
            val_ptr=d.val_ptr, col_val=d.col_val,
            pid=d.pid if d.pid is not None else np.zeros(0, np.int32),
            time=d.time if d.time is not None else np.zeros(0),
            has_offset=int(d.has_offset), has_intercept=int(d.has_intercept),
            prior=D.PRIOR_NONE, variance=1.0, weights=w if w is not None else np.zeros(0),
            tolerance=1e-6, convergence=D.CONV_GRADIENT,
            beta=fit.beta, log_likelihood=fit.log_likelihood, log_prior=fit.log_prior,
            iterations=fit.iterations, return_flag=fit.return_flag,
            tight_beta=tight.beta, tight_log_likelihood=tight.log_likelihood, tight_iterations=tight.iterations,
            newton_beta=nb, newton_log_likelihood=nll,
        )
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(f"{name:26s} K={d.K:4d} J={d.J} it={fit.iterations:3d} tight_it={tight.iterations:4d} "
              f"|tight-newton|={np.max(np.abs(tight.beta - nb)):.2e}")


# (fixture, prior, by_row, starting variance (<= 0: the normal-based default))
CV_AUTO_CASES = [("lr_laplace_small", D.PRIOR_LAPLACE, True, -1.0),
                 ("lr_c1", D.PRIOR_LAPLACE, True, -1.0),
                 ("clr_laplace", D.PRIOR_LAPLACE, False, -1.0),
                 ("cpr_normal", D.PRIOR_NORMAL, False, -1.0),
                 ("lr_zhang_oles", D.PRIOR_LAPLACE, True, 0.5),
                 ("cox_strata", D.PRIOR_LAPLACE, True, -1.0)]


def save_cv_auto():
    """cvauto_<case>.npz: the reference's auto-search cross-validation
    (AutoSearchCrossValidationDriver with UniModalSearch, one thread, cold
    starts, 10 folds, seed 123) on a fit fixture's data: the chosen variance,
    its predicted value and the points it tried."""
    for name, prior, by_row, start in CV_AUTO_CASES:
        d, _ = _load_fixture(name)
        bv, bval, tried = O.ref().cv_auto(d, prior, fold=10, n_reps=1, seed=123, by_row=by_row,
                                          starting_variance=start, reset_coefficients=True)
        np.savez_compressed(os.path.join(HERE, "cvauto_" + name + ".npz"), base=name, prior=prior, fold=10,
                            seed=123, by_row=int(by_row), starting_variance=start, best_variance=bv,
                            best_value=bval, tried=tried)
        print(f"cvauto_{name:20s} best={bv:.6g} value={bval:.6g} steps={len(tried)}")


def _load_fixture(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    data = D.CyclopsData(model=int(z["model"]), y=z["y"], col_format=z["col_format"], col_ptr=z["col_ptr"],
                         col_idx=z["col_idx"], val_ptr=z["val_ptr"], col_val=z["col_val"],
                         pid=z["pid"] if z["pid"].size else None, time=z["time"] if z["time"].size else None,
                         has_offset=bool(z["has_offset"]), has_intercept=bool(z["has_intercept"]))
    return data, z


def main(parts):
    if not O.have_ref():
        O.build()
    if "fits" in parts:
        for name, spec in cases().items():
            save_case(name, spec)
    if "cv" in parts:
        save_cv()
    if "bootstrap" in parts:
        save_bootstrap()
    if "ingest" in parts:
        save_ingest()
    if "swindle" in parts:
        save_swindle()
    if "profile" in parts:
        save_profile()
    if "small" in parts:
        save_small()
    if "cvauto" in parts:
        save_cv_auto()


if __name__ == "__main__":
    # python tests/golden/make_golden.py [fits] [cv] [bootstrap] [ingest] [swindle] [profile] [small] [cvauto]
    main(sys.argv[1:] or ["fits", "cv", "bootstrap", "ingest", "swindle", "profile", "small", "cvauto"])

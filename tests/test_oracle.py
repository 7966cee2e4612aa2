"""The CPU oracles, pinned against the golden fixtures made by the reference
engine (tests/golden/make_golden.py).  No GPU."""
import os

import numpy as np
import pytest

from conftest import golden_names, load_golden, profile_names, rel_err, small_names, swindle_names
from cyclops_b200 import data as D
from oracle import oracle as O


@pytest.mark.parametrize("name", golden_names())
def test_port_matches_reference_fixture(name):
    data, s = load_golden(name)
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]))
    fit = O.port().fit(data, int(s["prior"]), float(s["variance"]), control=ctl, weights=s["weights"])
    assert fit.iterations == int(s["iterations"])
    assert fit.return_flag == int(s["return_flag"])
    np.testing.assert_allclose(fit.beta, s["beta"], rtol=1e-12, atol=1e-14)
    assert abs(fit.log_likelihood - float(s["log_likelihood"])) <= 1e-12 * abs(float(s["log_likelihood"]))
    assert abs(fit.log_prior - float(s["log_prior"])) <= 1e-12 * max(1.0, abs(float(s["log_prior"])))


@pytest.mark.parametrize("name", golden_names())
def test_port_engine_probe_matches_reference_fixture(name):
    data, s = load_golden(name)
    g, h, xb, ll = O.port().probe(data, s["probe_beta"], int(s["prior"]), float(s["variance"]),
                                  weights=s["weights"])
    np.testing.assert_allclose(g, s["probe_gradient"], rtol=1e-12, atol=1e-10)
    np.testing.assert_allclose(h, s["probe_hessian"], rtol=1e-12, atol=1e-10)
    np.testing.assert_allclose(xb, s["probe_xbeta"], rtol=1e-13, atol=1e-14)
    assert rel_err(ll, float(s["probe_loglik"])) < 1e-12


def test_reference_and_port_agree_on_fresh_problem():
    if not O.have_ref():
        pytest.skip("reference engine not built here")
    d = D.synth_cox(K=1500, P=60, density=0.03, n_strata=3, seed=1234, ties=1)
    a = O.ref().fit(d, D.PRIOR_LAPLACE, 2.0)
    b = O.port().fit(d, D.PRIOR_LAPLACE, 2.0)
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(a.beta, b.beta)


def test_oracle_rejects_bad_model():
    d = D.synth_logistic(K=200, P=5, density=0.1, seed=3)
    d.model = 9
    with pytest.raises(RuntimeError):
        O.port().fit(d, D.PRIOR_NONE, 1.0)


def test_planted_mistake_is_caught():
    """A wrong Laplace rate in the oracle run changes the fit beyond the
    parity tolerance, so the comparison is sensitive."""
    data, s = load_golden("lr_laplace_small")
    bad = O.port().fit(data, int(s["prior"]), float(s["variance"]) * 1.01)
    assert np.max(rel_err(bad.beta[bad.beta != 0], s["beta"][bad.beta != 0], 1e-6)) > 1e-4


@pytest.mark.parametrize("name", swindle_names())
def test_port_swindle_matches_reference_fixture(name):
    """kktSwindle (CyclicCoordinateDescent.cpp:636-814): the restatement's
    active-set passes reproduce the reference's fit, iteration count and flag."""
    data, s = load_golden(name)
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]),
                         use_kkt_swindle=1)
    fit = O.port().fit(data, int(s["prior"]), float(s["variance"]), control=ctl, weights=s["weights"])
    assert fit.iterations == int(s["iterations"])
    assert fit.return_flag == int(s["return_flag"])
    np.testing.assert_allclose(fit.beta, s["beta"], rtol=1e-12, atol=1e-14)
    assert abs(fit.log_likelihood - float(s["log_likelihood"])) <= 1e-12 * abs(float(s["log_likelihood"]))


def test_swindle_fixtures_differ_from_plain_fits():
    """The swindle fixtures are not the plain fits renamed: the active-set
    passes end at a different point, within the convergence tolerance's reach
    of the plain fit (relative objective change below 1e-6 allows beta moves
    of a few hundredths on these problems)."""
    for name in swindle_names():
        _, sw = load_golden(name)
        _, plain = load_golden(name[len("swindle_"):])
        assert not np.array_equal(sw["beta"], plain["beta"])
        np.testing.assert_allclose(sw["beta"], plain["beta"], atol=5e-2)


def test_port_swindle_warm_start_and_pass_limit_match_reference():
    """A nonzero start on inactive columns (zeroed through updateXBeta) and a
    pass limit of 2 (MAX_ITERATIONS), against the reference run live."""
    if not O.have_ref():
        pytest.skip("reference engine not built here")
    data, s = load_golden("swindle_lr_laplace_small")
    start = np.where(np.arange(data.J) % 3 == 0, 0.05, 0.0)
    for max_it in (1000, 2):
        ctl = O.make_control(tolerance=1e-8, max_iterations=max_it, use_kkt_swindle=1)
        a = O.ref().fit(data, int(s["prior"]), float(s["variance"]), control=ctl, start=start)
        b = O.port().fit(data, int(s["prior"]), float(s["variance"]), control=ctl, start=start)
        assert (a.iterations, a.return_flag) == (b.iterations, b.return_flag)
        np.testing.assert_allclose(b.beta, a.beta, rtol=1e-12, atol=1e-14)
    assert b.return_flag == 2          # the pass limit was reached


@pytest.mark.parametrize("name", profile_names())
def test_port_profile_matches_reference_fixture(name):
    """profileModel (CcdInterface.cpp:262-420, one thread): the restated
    bracket + Brent root search over warm-started refits lands on the
    reference's bounds with the same number of refits."""
    data, s = load_golden(name)
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]),
                         use_kkt_swindle=int(s["swindle"]))
    lo, up, ev, fit = O.port().profile(data, s["columns"], int(s["prior"]), float(s["variance"]),
                                       float(s["threshold"]), bool(s["include_penalty"]), bool(s["override"]),
                                       control=ctl, weights=s["weights"])
    np.testing.assert_array_equal(ev, s["evaluations"])
    np.testing.assert_allclose(lo, s["lower"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(up, s["upper"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(fit.beta, s["beta"], rtol=1e-12, atol=1e-14)
    assert np.all(lo < fit.beta[s["columns"]]) and np.all(fit.beta[s["columns"]] < up)


def test_port_profile_rejects_regularized_column():
    data, s = load_golden("profile_lr_normal_weighted")
    with pytest.raises(RuntimeError, match="regularized"):
        O.port().profile(data, [3], int(s["prior"]), float(s["variance"]), override_no_regularization=False)


@pytest.mark.parametrize("name", profile_names())
def test_port_profile_points_match_reference_fixture(name):
    """evaluateProfileModel (CcdInterface.cpp:527-618, one thread)."""
    data, s = load_golden(name)
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]),
                         use_kkt_swindle=int(s["swindle"]))
    vals = O.port().profile_points(data, int(s["point_column"]), s["points"], int(s["prior"]),
                                   float(s["variance"]), bool(s["include_penalty"]), control=ctl,
                                   weights=s["weights"])
    np.testing.assert_allclose(vals, s["point_values"], rtol=1e-13)
    assert np.argmax(vals) in (3, 4, 5)            # the points straddle the estimate


@pytest.mark.parametrize("name", small_names())
def test_newton_mle_agrees_with_reference_on_small_designs(name):
    """The second, independent check: a NumPy Newton-Raphson MLE of the same
    likelihood (oracle/newton.py) lands where the reference engine's CCD
    does when run until its log likelihood stops changing."""
    from oracle import newton
    data, s = load_golden(name)
    nb, nll = newton.newton_fit(data, s["weights"])
    np.testing.assert_allclose(nb, s["newton_beta"], rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(s["tight_beta"], nb, rtol=2e-6, atol=2e-6)
    assert abs(float(s["tight_log_likelihood"]) - nll) <= 1e-11 * abs(nll)


@pytest.mark.parametrize("name", small_names())
def test_port_matches_reference_on_small_designs(name):
    data, s = load_golden(name)
    ex = [1 if data.has_offset else 0] if data.has_intercept else []
    fit = O.port().fit(data, D.PRIOR_NONE, 1.0, control=O.make_control(), exclude=ex, weights=s["weights"])
    assert (fit.iterations, fit.return_flag) == (int(s["iterations"]), int(s["return_flag"]))
    np.testing.assert_allclose(fit.beta, s["beta"], rtol=1e-12, atol=1e-14)
    tight = O.port().fit(data, D.PRIOR_NONE, 1.0, exclude=ex, weights=s["weights"],
                         control=O.make_control(tolerance=1e-17, convergence_type=D.CONV_MITTAL,
                                                max_iterations=100000))
    assert tight.iterations == int(s["tight_iterations"])
    np.testing.assert_allclose(tight.beta, s["tight_beta"], rtol=1e-12, atol=1e-14)


def test_small_design_properties():
    """The reference's own invariances on its small designs: zero weight is
    removal (test-smallCox.R), and dense, sparse and indicator columns give
    the same fit (test-smallBernoulli.R, test-smallPoisson.R)."""
    for a, b in [("small_cox_zero_weights", "small_cox_failties_strata"), ("small_lr_dense", "small_lr_sparse"),
                 ("small_pr_dense", "small_pr_indicator")]:
        _, sa = load_golden(a)
        _, sb = load_golden(b)
        np.testing.assert_allclose(sa["tight_beta"], sb["tight_beta"], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(sa["newton_beta"], sb["newton_beta"], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("name,cols", [("small_pr_dense", [0, 1, 3]), ("small_lr_dense", [0, 1]),
                                       ("small_cox_failties_risk", [0, 1]), ("small_clr_infert", [0, 1])])
def test_profile_bounds_agree_with_newton_profile(name, cols):
    """The profile search (bracket + Brent at tolerance 1e-3, restated from
    profileModel) against roots of the Newton profile log likelihood found
    to 1e-12: within the search's 1e-3 tolerance, as R's confint is."""
    from scipy.optimize import brentq
    from oracle import newton
    data, s = load_golden(name)
    thr = 1.920729410347062
    ctl = O.make_control(tolerance=1e-10, convergence_type=D.CONV_MITTAL, max_iterations=100000)
    lo, up, ev, fit = O.port().profile(data, cols, D.PRIOR_NONE, 1.0, thr, False, True, control=ctl,
                                       weights=s["weights"])
    nb, nll = newton.newton_fit(data, s["weights"])
    with np.errstate(over="ignore", invalid="ignore"):
        for i, j in enumerate(cols):
            f = lambda x: newton.newton_fit(data, s["weights"], fixed={j: x})[1] - (nll - thr)
            ru = brentq(f, nb[j], up[i] + 0.5 * (up[i] - nb[j]), xtol=1e-12)
            rl = brentq(f, lo[i] - 0.5 * (nb[j] - lo[i]), nb[j], xtol=1e-12)
            assert abs(up[i] - ru) < 1e-3 and abs(lo[i] - rl) < 1e-3, (j, up[i] - ru, lo[i] - rl)


def test_port_fixed_coefficients_match_reference():
    """fixedCoefficients (R/ModelFit.R:205-214 -> setFixedBeta): the Dobson
    design with outcome3 and treatment3 fixed as test-smallPoisson.R fixes
    them (at 0, and at other starts), and a Laplace fit with two fixed
    columns with and without the KKT swindle, against the reference run live."""
    if not O.have_ref():
        pytest.skip("reference engine not built here")
    data, s = load_golden("small_pr_dense")
    for start in (np.zeros(5), np.array([0.0, 0.3, 0.0, -0.2, 0.0])):
        a = O.ref().fit(data, D.PRIOR_NONE, 1.0, exclude=[0], start=start, fixed=[1, 3])
        b = O.port().fit(data, D.PRIOR_NONE, 1.0, exclude=[0], start=start, fixed=[1, 3])
        assert a.beta[1] == start[1] and a.beta[3] == start[3]
        assert a.iterations == b.iterations
        np.testing.assert_allclose(b.beta, a.beta, rtol=1e-12, atol=1e-14)
    data, s = load_golden("lr_laplace_small")
    start = np.zeros(data.J)
    start[[3, 7]] = [0.4, -0.25]
    for sw in (0, 1):
        ctl = O.make_control(use_kkt_swindle=sw)
        a = O.ref().fit(data, D.PRIOR_LAPLACE, float(s["variance"]), control=ctl, start=start, fixed=[3, 7])
        b = O.port().fit(data, D.PRIOR_LAPLACE, float(s["variance"]), control=ctl, start=start, fixed=[3, 7])
        assert a.iterations == b.iterations
        np.testing.assert_allclose(b.beta, a.beta, rtol=1e-12, atol=1e-14)


def _float_rounded(data):
    """The data as ModelData<float> holds it: outcomes, times and values
    rounded to float, widened back to double."""
    from cyclops_b200.data import CyclopsData
    r = lambda a: None if a is None else np.asarray(a, np.float32).astype(np.float64)
    return CyclopsData(model=data.model, y=r(data.y), col_format=data.col_format, col_ptr=data.col_ptr,
                       col_idx=data.col_idx, val_ptr=data.val_ptr, col_val=r(data.col_val), pid=data.pid,
                       time=r(data.time), has_offset=data.has_offset, has_intercept=data.has_intercept)


def ref_fit_fp32(lib, data, s, device):
    """ref_fit_fp32 of a harness library: the reference's CCD on
    ModelData<float> (device 0: its float CPU engine; 1: the CUDA engine)."""
    import ctypes as C
    lib.ref_fit_fp32.argtypes = [C.POINTER(O.Problem), C.POINTER(O.Control), C.c_void_p, C.POINTER(O.Result),
                                 C.c_int]
    lib.ref_last_error.restype = C.c_char_p
    p, keep = O.make_problem(data, int(s["prior"]), float(s["variance"]), None, s["weights"])
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]))
    beta = np.zeros(data.J)
    r = O.Result(beta=beta.ctypes.data)
    assert lib.ref_fit_fp32(C.byref(p), C.byref(ctl), None, C.byref(r), device) == 0, lib.ref_last_error()
    return O.Fit(beta, r.log_likelihood, r.log_prior, r.iterations, r.return_flag)


def test_reference_float_data_fit():
    """The reference's own FP32 path (floatingPoint = 32) on the binomial bid
    design of test-floatingPoint.R fits the FP64 coefficients to the
    reference test's own bound (1e-3, against glm there)."""
    import ctypes as C
    if not O.have_ref():
        pytest.skip("reference engine not built")
    data, s = load_golden("small_lr_dense")
    lib = C.CDLL(os.path.join(O.REF_DIR, "libcyclops_ref.so"))
    f32 = ref_fit_fp32(lib, data, s, 0)
    assert f32.return_flag == 0
    np.testing.assert_allclose(f32.beta, s["beta"], rtol=1e-3)

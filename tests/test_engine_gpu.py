"""Per-coordinate engine (the AbstractModelSpecifics surface) on the GPU
against the reference engine's outputs at the same coefficients."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, rel_err

pytestmark = pytest.mark.gpu


def _engine(data, weights):
    from cyclops_b200 import api
    ds = api.Dataset(data)
    e = api.Engine(ds)
    use = weights is not None
    e.set_weights(weights, use_cv=use)
    e.compute_fixed_terms_in_log_likelihood(use)
    e.compute_fixed_terms_in_gradient_and_hessian(use)
    return ds, e, use


@pytest.mark.parametrize("name", golden_names())
def test_engine_matches_reference_at_fixed_beta(cuda_lib, name):
    data, s = load_golden(name)
    ds, e, use = _engine(data, s["weights"])
    e.compute_xbeta(s["probe_beta"], use)
    e.compute_remaining_statistics(use)
    xb = e.get_xbeta()
    np.testing.assert_allclose(xb, s["probe_xbeta"], rtol=1e-14, atol=1e-14)
    ll = e.get_log_likelihood(use)
    assert rel_err(ll, float(s["probe_loglik"])) < 1e-10, (ll, float(s["probe_loglik"]))
    g = np.zeros(data.J)
    h = np.zeros(data.J)
    for j in range(data.J):
        e.compute_numerator_for_gradient(j, use)
        g[j], h[j] = e.compute_gradient_and_hessian(j, use)
    gr, hr = s["probe_gradient"], s["probe_hessian"]
    scale = np.abs(hr) + 1.0
    assert np.all(np.abs(g - gr) <= 1e-9 * (np.abs(gr) + scale)), np.max(np.abs(g - gr) / (np.abs(gr) + scale))
    assert np.all(np.abs(h - hr) <= 1e-9 * scale), np.max(np.abs(h - hr) / scale)


@pytest.mark.parametrize("name", ["lr_laplace_small", "pr_laplace_weighted", "clr_laplace", "cox_strata",
                                  "cox_ties_weighted"])
def test_update_then_gradient_tracks_oracle(cuda_lib, name):
    """A few coordinate updates through the engine, then the state matches the
    oracle evaluated at the moved coefficients."""
    from oracle import oracle as O
    data, s = load_golden(name)
    ds, e, use = _engine(data, s["weights"])
    beta = np.array(s["probe_beta"], float)
    e.compute_xbeta(beta, use)
    e.compute_remaining_statistics(use)
    rng = np.random.default_rng(3)
    first = 1 if data.has_offset else 0
    for j in rng.choice(np.arange(first, data.J), size=min(8, data.J - first), replace=False):
        d = float(rng.normal(0, 0.1))
        e.update_xbeta(d, int(j), use)
        beta[j] += d
    g_ref, h_ref, xb_ref, ll_ref = O.port().probe(data, beta, int(s["prior"]), float(s["variance"]),
                                                  weights=s["weights"])
    np.testing.assert_allclose(e.get_xbeta(), xb_ref, rtol=1e-12, atol=1e-12)
    assert rel_err(e.get_log_likelihood(use), ll_ref) < 1e-9
    for j in range(0, data.J, max(1, data.J // 25)):
        e.compute_numerator_for_gradient(j, use)
        g, h = e.compute_gradient_and_hessian(j, use)
        sc = abs(h_ref[j]) + 1.0
        assert abs(g - g_ref[j]) <= 1e-8 * (abs(g_ref[j]) + sc)
        assert abs(h - h_ref[j]) <= 1e-8 * sc


def test_predictive_loglik_matches_oracle(cuda_lib):
    from oracle import oracle as O
    for name in ("lr_laplace_small", "pr_offset_normal", "cox_laplace"):
        data, s = load_golden(name)
        ds, e, use = _engine(data, None)
        e.compute_xbeta(s["beta"])
        e.compute_remaining_statistics()
        held = (np.arange(data.K) % 3 == 0).astype(float)
        got = e.get_predictive_log_likelihood(held)
        want = O.port().predictive_loglik(data, s["beta"], held)
        assert rel_err(got, want) < 1e-10, (name, got, want)


def test_predictive_estimates_match_reference(cuda_lib):
    """getPredictiveEstimates (ModelSpecifics.hpp:693-707): the logistic
    probability, the Poisson mean, or xbeta, on the rows with nonzero weight;
    the caller's other entries stay as they were."""
    from cyclops_b200 import _native as N
    from oracle import oracle as O
    if not O.have_ref():
        pytest.skip("reference engine not built here")
    for name in ("lr_laplace_small", "pr_offset_normal", "clr_laplace", "cox_laplace"):
        data, s = load_golden(name)
        ds, e, use = _engine(data, None)
        e.compute_xbeta(s["beta"])
        e.compute_remaining_statistics()
        w = (np.arange(data.K) % 4 != 0).astype(float)
        want = O.ref().predictive_estimates(data, s["beta"], w, fill=-7.0)
        y = np.full(data.K, -7.0)
        N.check(N.lib().cyc_engine_get_predictive_estimates(e.handle, y.ctypes.data, w.ctypes.data))
        np.testing.assert_allclose(y, want, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(e.get_predictive_estimates(), O.ref().predictive_estimates(data, s["beta"]),
                                   rtol=1e-12, atol=1e-14)


def test_gradient_before_statistics_is_a_state_error(cuda_lib):
    from cyclops_b200 import api, _native
    data, s = load_golden("lr_laplace_small")
    e = api.Engine(api.Dataset(data))
    with pytest.raises(_native.CyclopsError) as ei:
        e.compute_gradient_and_hessian(1)
    assert ei.value.status == 5

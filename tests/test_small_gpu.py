"""The tiny designs of the reference's own tests (test-smallCox.R,
test-smallBernoulli.R, test-smallPoisson.R: Cox with and without ties,
strata and zero weights; dense and sparse logistic; dense and indicator
Poisson) fitted unpenalised on the GPU, against the reference engine's fits
and the independent Newton MLE stored with them."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, exclude_for, load_golden, small_names
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu

ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libcyclops_ref_cuda.so")


def _fit(data, s, **ctl):
    from cyclops_b200 import api
    prior = api.PriorSpec(D.PRIOR_NONE, 1.0, exclude_for(data))
    return api.fit_cyclops_model(data, prior, api.create_control(**ctl), weights=s["weights"])


@pytest.mark.parametrize("name", small_names())
def test_small_design_default_control(cuda_lib, name):
    data, s = load_golden(name)
    fit = _fit(data, s)
    assert fit.return_flag == int(s["return_flag"])
    assert fit.iterations == int(s["iterations"])
    np.testing.assert_allclose(fit.beta, s["beta"], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("name", small_names())
def test_small_design_converged_to_newton_mle(cuda_lib, name):
    """Run until the log likelihood stops changing: the MLE of the Newton
    restatement (beta 2e-6, log likelihood 1e-11 relative)."""
    data, s = load_golden(name)
    fit = _fit(data, s, tolerance=1e-17, convergence_type="mittal", max_iterations=100000)
    np.testing.assert_allclose(fit.beta, s["newton_beta"], rtol=2e-6, atol=2e-6)
    nll = float(s["newton_log_likelihood"])
    assert abs(fit.log_likelihood - nll) <= 1e-11 * abs(nll)


@pytest.mark.skipif(not os.path.exists(ADAPTER), reason="adapter harness not built (needs the reference sources)")
@pytest.mark.parametrize("name", ["small_cox_failties_risk", "small_cox_zero_weights", "small_lr_sparse",
                                  "small_pr_indicator"])
def test_small_design_reference_ccd_on_cuda_engine(cuda_lib, name):
    from oracle import oracle as O
    data, s = load_golden(name)
    lib = C.CDLL(ADAPTER)
    lib.ref_fit_device.argtypes = [C.POINTER(O.Problem), C.POINTER(O.Control), C.c_void_p,
                                   C.POINTER(O.Result), C.c_int]
    lib.ref_last_error.restype = C.c_char_p
    p, keep = O.make_problem(data, D.PRIOR_NONE, 1.0, None, s["weights"])
    ctl = O.make_control()
    beta = np.zeros(data.J)
    r = O.Result(beta=beta.ctypes.data)
    assert lib.ref_fit_device(C.byref(p), C.byref(ctl), None, C.byref(r), 1) == 0, lib.ref_last_error()
    assert r.iterations == int(s["iterations"])
    np.testing.assert_allclose(beta, s["beta"], rtol=1e-6, atol=1e-9)

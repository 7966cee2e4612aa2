"""Fixed coefficients on the GPU (cyc_fit_spec.fixed: fitCyclopsModel's
fixedCoefficients, R/ModelFit.R:205-214 -> setFixedBeta) against the
restatement oracle, which matches the reference on the same cases."""
import numpy as np
import pytest

from conftest import exclude_for, load_golden
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu


def test_fixed_dobson_single_fit(cuda_lib):
    """test-smallPoisson.R's fixed-beta case: outcome3 and treatment3 held at
    their starts while the rest refit."""
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden("small_pr_dense")
    prior = api.PriorSpec(D.PRIOR_NONE, 1.0, exclude_for(data))
    for start in (np.zeros(5), np.array([0.0, 0.3, 0.0, -0.2, 0.0])):
        want = O.port().fit(data, D.PRIOR_NONE, 1.0, exclude=[0], start=start, fixed=[1, 3])
        mask = np.array([False, True, False, True, False])
        got = api.fit_cyclops_model(data, prior, api.create_control(), starting_coefficients=start,
                                    fixed_coefficients=mask)
        assert got.beta[1] == start[1] and got.beta[3] == start[3]
        assert got.iterations == want.iterations
        np.testing.assert_allclose(got.beta, want.beta, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("swindle", [False, True])
def test_fixed_laplace_single_fit(cuda_lib, swindle):
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden("lr_laplace_small")
    start = np.zeros(data.J)
    start[[3, 7]] = [0.4, -0.25]
    octl = O.make_control(tolerance=1e-10, use_kkt_swindle=int(swindle))
    want = O.port().fit(data, D.PRIOR_LAPLACE, float(s["variance"]), control=octl, start=start, fixed=[3, 7])
    prior = api.PriorSpec(D.PRIOR_LAPLACE, float(s["variance"]), exclude_for(data))
    got = api.fit_cyclops_model(data, prior, api.create_control(tolerance=1e-10, use_kkt_swindle=swindle),
                                starting_coefficients=start, fixed_coefficients=[3, 7])
    assert got.iterations == want.iterations
    np.testing.assert_array_equal(got.beta != 0, want.beta != 0)
    np.testing.assert_allclose(got.beta, want.beta, rtol=1e-6, atol=1e-9)


def test_fixed_batched_fits(cuda_lib):
    """Four fits of one batch share the fixed columns, each at its own start."""
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden("lr_laplace_small")
    variances = [D.laplace_variance(l) for l in (0.5, 1.0, 2.0, 4.0)]
    starts = []
    for f in range(4):
        st = np.zeros(data.J)
        st[[3, 7]] = [0.1 * (f + 1), -0.05 * f]
        starts.append(st)
    prior = api.PriorSpec(D.PRIOR_LAPLACE, 1.0, exclude_for(data))
    ctl = api.create_control(tolerance=1e-10)
    got = api.batch_fit(data, prior, variances, control=ctl, starts=starts, fixed_coefficients=[3, 7])
    for f in range(4):
        want = O.port().fit(data, D.PRIOR_LAPLACE, variances[f], control=O.make_control(tolerance=1e-10),
                            start=starts[f], fixed=[3, 7])
        assert got[f].beta[3] == starts[f][3] and got[f].beta[7] == starts[f][7]
        assert got[f].iterations == want.iterations
        np.testing.assert_allclose(got[f].beta, want.beta, rtol=1e-6, atol=1e-9)
    # fits of one batch with different fixed sets are refused
    import ctypes as C
    from cyclops_b200 import _native as N
    ds = api.Dataset(data)
    p, keep = api._prior_struct(data, prior)
    a, b = np.array([3], np.int32), np.array([7], np.int32)
    specs = (N.FitSpec * 2)(N.FitSpec(variance=1.0, fixed=a.ctypes.data, n_fixed=1),
                            N.FitSpec(variance=1.0, fixed=b.ctypes.data, n_fixed=1))
    outs = np.zeros((2, data.J))
    res = (N.FitResult * 2)(N.FitResult(beta=outs[0].ctypes.data), N.FitResult(beta=outs[1].ctypes.data))
    c = api._control_struct(ctl)
    with pytest.raises(N.CyclopsError) as ei:
        N.check(N.lib().cyc_batch_fit(ds.handle, C.byref(p), specs, 2, C.byref(c), res))
    assert ei.value.status == 4

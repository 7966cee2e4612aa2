"""Profile-likelihood bounds on the GPU (cyc_profile_bounds: each refit a
device-resident CCD warm-started from the last) against the reference's
CcdInterface::profileModel (src/cyclops/CcdInterface.cpp:262-420, one
thread): the profile_* fixtures the reference made, and the restatement
oracle on a new seeded problem."""
import numpy as np
import pytest

from conftest import exclude_for, load_golden, profile_names
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu

# the root search stops within 1e-3 (RZeroIn tolerance); refits agree to
# ~1e-9, so the bounds agree far inside that
BOUND_ATOL = 1e-6


def _profile(data, s, columns=None, **kw):
    from cyclops_b200 import api
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    ctl = api.create_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]),
                             use_kkt_swindle=bool(s["swindle"]))
    return api.profile_bounds(data, s["columns"] if columns is None else columns, prior, ctl,
                              threshold=float(s["threshold"]), include_penalty=bool(s["include_penalty"]),
                              override_no_regularization=bool(s["override"]), weights=s["weights"], **kw)


@pytest.mark.parametrize("name", profile_names())
def test_profile_matches_reference_fixture(cuda_lib, name):
    data, s = load_golden(name)
    pb = _profile(data, s)
    np.testing.assert_array_equal(pb.evaluations, s["evaluations"])
    np.testing.assert_allclose(pb.lower, s["lower"], rtol=0, atol=BOUND_ATOL)
    np.testing.assert_allclose(pb.upper, s["upper"], rtol=0, atol=BOUND_ATOL)
    np.testing.assert_allclose(pb.fit.beta, s["beta"], rtol=1e-6, atol=1e-9)


def test_profile_new_problem_matches_oracle(cuda_lib):
    """A fresh seeded Poisson problem with an offset, profiled on every
    unregularized column under a normal prior with the override."""
    from oracle import oracle as O
    d = D.synth_poisson(K=2500, P=40, per_row=5, n_dense=2, n_true=10, seed=77)
    cols = [1, 2, 5, 11]
    thr = 1.920729410347062
    ctl = O.make_control(tolerance=1e-7)
    lo, up, ev, fit = O.port().profile(d, cols, D.PRIOR_NORMAL, 2.0, thr, True, True, control=ctl)
    s = dict(prior=D.PRIOR_NORMAL, variance=2.0, tolerance=1e-7, convergence=D.CONV_GRADIENT, swindle=0,
             columns=np.asarray(cols), threshold=thr, include_penalty=1, override=1, weights=None)
    pb = _profile(d, s)
    np.testing.assert_array_equal(pb.evaluations, ev)
    np.testing.assert_allclose(pb.lower, lo, rtol=0, atol=BOUND_ATOL)
    np.testing.assert_allclose(pb.upper, up, rtol=0, atol=BOUND_ATOL)


def test_profile_rejects_regularized_and_offset(cuda_lib):
    from cyclops_b200 import _native
    data, s = load_golden("profile_lr_normal_weighted")
    s = dict(s, override=0)
    with pytest.raises(_native.CyclopsError) as ei:
        _profile(data, s, columns=[3])
    assert ei.value.status == 1 and "regularized" in str(ei.value)
    data, s = load_golden("profile_pr_offset_normal")
    with pytest.raises(_native.CyclopsError) as ei:
        _profile(data, s, columns=[0])
    assert ei.value.status == 1


@pytest.mark.parametrize("name", profile_names())
def test_profile_points_match_reference_fixture(cuda_lib, name):
    """getCyclopsProfileLogLikelihood (evaluateProfileModel, one thread)."""
    from cyclops_b200 import api
    data, s = load_golden(name)
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    ctl = api.create_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]),
                             use_kkt_swindle=bool(s["swindle"]))
    vals = api.profile_log_likelihood(data, int(s["point_column"]), s["points"], prior, ctl,
                                      include_penalty=bool(s["include_penalty"]), weights=s["weights"])
    np.testing.assert_allclose(vals, s["point_values"], rtol=1e-9)


@pytest.mark.parametrize("name", ["profile_lr_normal_weighted", "profile_clr_normal_weighted",
                                  "profile_pr_offset_normal", "profile_lr_flat"])
def test_profile_points_batched_match_oracle(cuda_lib, name):
    """All points refit together in the batch kernel (column held fixed,
    each from the mode), against the oracle's one-thread chain, both
    converged tightly (Mittal 1e-11): the values agree to 1e-9 relative."""
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden(name)
    col = int(s["point_column"])
    pts = s["points"]
    octl = O.make_control(tolerance=1e-11, convergence_type=D.CONV_MITTAL, max_iterations=5000)
    want = O.port().profile_points(data, col, pts, int(s["prior"]), float(s["variance"]),
                                   bool(s["include_penalty"]), control=octl, weights=s["weights"])
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    ctl = api.create_control(tolerance=1e-11, convergence_type=D.CONV_MITTAL, max_iterations=5000)
    got = api.profile_log_likelihood(data, col, pts, prior, ctl, include_penalty=bool(s["include_penalty"]),
                                     weights=s["weights"], batched=True)
    np.testing.assert_allclose(got, want, rtol=1e-9)

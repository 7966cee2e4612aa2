"""Host-side pieces of the Python API that need no GPU: control and prior
mapping onto the C structs, the fixed-coefficient argument, the profile
threshold."""
import math

import numpy as np
import pytest

from cyclops_b200 import api
from cyclops_b200 import data as D


def test_control_maps_every_field():
    c = api.create_control(tolerance=1e-8, max_iterations=77, convergence_type="lange", initial_bound=3.0,
                           max_bound_count=4, precision="mixed", polish_tolerance=1e-3, use_kkt_swindle=True)
    s = api._control_struct(c)
    assert (s.tolerance, s.max_iterations, s.convergence_type, s.initial_bound, s.max_bound_count, s.precision,
            s.polish_tolerance, s.use_kkt_swindle) == (1e-8, 77, D.CONV_LANGE, 3.0, 4, 1, 1e-3, 1)
    assert api._control_struct(api.create_control()).use_kkt_swindle == 0


def test_fixed_coefficients_argument():
    assert api._fixed_columns(None, 5) is None
    assert api._fixed_columns([], 5) is None
    np.testing.assert_array_equal(api._fixed_columns([False, True, False, True, False], 5), [1, 3])
    np.testing.assert_array_equal(api._fixed_columns([4, 0], 5), [4, 0])
    with pytest.raises(ValueError):
        api._fixed_columns([True, False], 5)


def test_profile_threshold_is_half_the_chi_square_quantile():
    # qchisq(0.95, 1) / 2 and qchisq(0.9, 1) / 2
    assert abs(api.profile_threshold(0.95) - 1.920729410347062) < 1e-12
    assert abs(api.profile_threshold(0.90) - 2.705543454095404 / 2) < 1e-12
    with pytest.raises(ValueError):
        api.profile_threshold(0.999)


def test_intercept_is_excluded_from_the_prior_unless_forced():
    d = D.synth_logistic(K=50, P=3, density=0.2, n_true=1, seed=2)
    assert api._exclude_for(d, api.create_prior("laplace", 1.0)) == [0]
    assert api._exclude_for(d, api.create_prior("laplace", 1.0, force_intercept=True)) == []
    assert api._exclude_for(d, api.create_prior("none")) == []
    assert math.isclose(D.laplace_variance(0.1), 200.0)

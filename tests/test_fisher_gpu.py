"""Fisher information and asymptotic variance on the GPU
(cyc_engine_fisher_information) against the reference's
CyclicCoordinateDescent::computeFisherInformation at the same coefficients,
and the reference's own CCD asking for it through the CUDA adapter."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import ROOT, load_golden
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu

ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libcyclops_ref_cuda.so")
CASES = ["lr_laplace_small", "lr_normal_weighted", "lr_c1", "pr_laplace_weighted", "pr_offset_normal",
         "clr_laplace", "clr_normal_weighted", "cpr_normal"]
RTOL = 1e-11      # sums in a different order than the reference's sequential ones


def _columns(data, beta, most=24):
    cols = [j for j in range(data.J) if beta[j] != 0.0 and not (data.has_offset and j == 0)]
    return cols[:most]


@pytest.mark.parametrize("name", CASES)
def test_fisher_matches_reference(cuda_lib, name):
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden(name)
    beta = s["beta"]
    cols = _columns(data, beta)
    ref = O.ref().fisher(data, beta, cols)
    eng = api.Engine(api.Dataset(data))
    eng.compute_xbeta(beta)
    eng.compute_remaining_statistics()
    got = eng.fisher_information(cols)
    scale = np.sqrt(np.outer(np.abs(np.diag(ref)), np.abs(np.diag(ref)))) + 1e-300
    assert np.max(np.abs(got - ref) / scale) < RTOL
    np.testing.assert_array_equal(got, got.T)


@pytest.mark.parametrize("name", ["lr_laplace_small", "clr_laplace", "pr_laplace_weighted", "cpr_normal"])
def test_asymptotic_variance(cuda_lib, name):
    """getAsymptoticVariance: the inverse over the non-fixed (and, under a
    Laplace prior, non-zero) columns.  The cases have well-conditioned
    information matrices (condition number below 1e4, checked), so the
    inverses agree as closely as the matrices do."""
    from cyclops_b200 import api
    from oracle import oracle as O
    data, s = load_golden(name)
    beta = s["beta"]
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]))
    av = api.asymptotic_variance(data, beta, prior)
    want = [j for j in range(data.J) if not (data.has_offset and j == 0)
            and (int(s["prior"]) != D.PRIOR_LAPLACE or beta[j] != 0.0)]
    np.testing.assert_array_equal(av.columns, want)
    ref_fisher = O.ref().fisher(data, beta, want)
    assert np.linalg.cond(ref_fisher) < 1e4
    ref = np.linalg.inv(ref_fisher)
    scale = np.sqrt(np.outer(np.diag(ref), np.diag(ref)))          # covariance scale of each entry
    assert np.max(np.abs(av.variance - ref) / scale) < 1e-9
    assert np.all(av.standard_errors > 0)


@pytest.mark.skipif(not os.path.exists(ADAPTER), reason="adapter harness not built (needs the reference sources)")
@pytest.mark.parametrize("name", ["lr_laplace_small", "clr_laplace"])
def test_reference_ccd_fisher_through_adapter(cuda_lib, name):
    from oracle import oracle as O
    data, s = load_golden(name)
    beta = s["beta"]
    cols = _columns(data, beta, most=10)
    lib = C.CDLL(ADAPTER)
    lib.ref_fisher.argtypes = [C.POINTER(O.Problem), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int]
    lib.ref_last_error.restype = C.c_char_p
    p, keep = O.make_problem(data, 1, 1.0, None, None)
    b = np.ascontiguousarray(beta, np.float64)
    cc = np.ascontiguousarray(cols, np.int32)
    out = np.zeros((len(cols), len(cols)))
    assert lib.ref_fisher(C.byref(p), b.ctypes.data, cc.ctypes.data, len(cols), out.ctypes.data, 1) == 0, \
        lib.ref_last_error()
    ref = O.ref().fisher(data, beta, cols)
    scale = np.sqrt(np.outer(np.abs(np.diag(ref)), np.abs(np.diag(ref)))) + 1e-300
    assert np.max(np.abs(out - ref) / scale) < RTOL


def test_fisher_unsupported(cuda_lib):
    from cyclops_b200 import api, _native
    data, s = load_golden("cox_laplace")
    eng = api.Engine(api.Dataset(data))
    with pytest.raises(_native.CyclopsError) as ei:
        eng.fisher_information([0, 1])
    assert ei.value.status == 4
    data, s = load_golden("lr_laplace_small")
    eng = api.Engine(api.Dataset(data))
    with pytest.raises(_native.CyclopsError) as ei:
        eng.fisher_information([0, 1], use_cv=True)
    assert ei.value.status == 4

"""Device-resident CCD (cyc_fit) and the drop-in adapter (the reference's
own CyclicCoordinateDescent driving the CUDA engine) against the reference."""
import os
import types

import numpy as np
import pytest

from conftest import ROOT, assert_contract, exclude_for, golden_fit, golden_names, load_golden
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu


def _gpu_fit(data, s, tolerance=None, convergence=None, max_iterations=1000):
    from cyclops_b200 import api
    prior = api.PriorSpec(int(s["prior"]), float(s["variance"]), exclude_for(data))
    ctl = api.create_control(tolerance=float(s["tolerance"]) if tolerance is None else tolerance,
                             convergence_type=int(s["convergence"]) if convergence is None else convergence,
                             max_iterations=max_iterations)
    return api.fit_cyclops_model(data, prior, ctl, weights=s["weights"])


@pytest.mark.parametrize("name", golden_names())
def test_device_fit_matches_reference_fit(cuda_lib, name):
    """Same prior, tolerance and convergence rule as the reference run: the
    precision contract, cycle for cycle."""
    data, s = load_golden(name)
    assert_contract(_gpu_fit(data, s), golden_fit(s), what=name)


@pytest.mark.parametrize("name", ["lr_c1", "pr_offset_normal", "clr_laplace", "cpr_normal",
                                  "cox_laplace", "cox_strata", "cox_ties_weighted", "lr_normal_weighted"])
def test_device_fit_tight_contract(cuda_lib, name):
    """Both sides converged tightly (tolerance 1e-12): beta 1e-6 relative,
    log likelihood 1e-9 relative, identical zero pattern."""
    from oracle import oracle as O
    data, s = load_golden(name)
    ctl = O.make_control(tolerance=1e-12, convergence_type=D.CONV_MITTAL, max_iterations=5000)
    ref = O.port().fit(data, int(s["prior"]), float(s["variance"]), control=ctl, weights=s["weights"])
    fit = _gpu_fit(data, s, tolerance=1e-12, convergence=D.CONV_MITTAL, max_iterations=5000)
    assert_contract(fit, ref, what=name)


ADAPTER = os.path.join(ROOT, "oracle", "_ref", "libcyclops_ref_cuda.so")


@pytest.mark.skipif(not os.path.exists(ADAPTER), reason="adapter harness not built (needs the reference sources)")
@pytest.mark.parametrize("name", golden_names())
def test_reference_ccd_drives_cuda_engine(cuda_lib, name):
    """The reference's CyclicCoordinateDescent, unchanged, with the engine
    replaced through CudaModelSpecifics: same iterations and coefficients."""
    import ctypes as C
    from oracle import oracle as O
    data, s = load_golden(name)
    lib = C.CDLL(ADAPTER)
    lib.ref_fit_device.argtypes = [C.POINTER(O.Problem), C.POINTER(O.Control), C.c_void_p,
                                   C.POINTER(O.Result), C.c_int]
    lib.ref_last_error.restype = C.c_char_p
    p, keep = O.make_problem(data, int(s["prior"]), float(s["variance"]), None, s["weights"])
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]))
    beta = np.zeros(data.J)
    r = O.Result(beta=beta.ctypes.data)
    rc = lib.ref_fit_device(C.byref(p), C.byref(ctl), None, C.byref(r), 1)
    assert rc == 0, lib.ref_last_error()
    got = types.SimpleNamespace(beta=beta, log_likelihood=r.log_likelihood, iterations=r.iterations,
                                return_flag=r.return_flag)
    assert_contract(got, golden_fit(s), what=name)


@pytest.mark.skipif(not os.path.exists(ADAPTER), reason="adapter harness not built (needs the reference sources)")
@pytest.mark.parametrize("name", ["small_lr_dense", "lr_normal_weighted", "pr_offset_normal", "cox_laplace",
                                  "clr_laplace"])
def test_reference_ccd_drives_cuda_engine_on_float_data(cuda_lib, name):
    """ModelData<float> (the reference's floatingPoint = 32) behind the
    drop-in: the adapter widens the float values to double at upload, so the
    fit is the reference FP64 engine's on the float-rounded data, under the
    precision contract."""
    import ctypes as C
    from oracle import oracle as O
    from test_oracle import _float_rounded, ref_fit_fp32
    data, s = load_golden(name)
    got = ref_fit_fp32(C.CDLL(ADAPTER), data, s, 1)
    ctl = O.make_control(tolerance=float(s["tolerance"]), convergence_type=int(s["convergence"]))
    want = O.ref().fit(_float_rounded(data), int(s["prior"]), float(s["variance"]), control=ctl,
                       weights=s["weights"])
    assert_contract(got, want, what=name)

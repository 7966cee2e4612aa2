"""The allocation-free gradient/Hessian entry point, called through the C ABI.

Some callers cannot let the library allocate device memory (they manage the
GPU's memory in their own pool, or cannot take the synchronisation an
allocation implies); cyc_gradient_hessian_noalloc serves them from a fixed
scratch area compiled into the library.  This test gives it caller-owned
device buffers and checks its (gradient, Hessian) against
cyc_engine_compute_gradient_and_hessian on the same state, twice in a row
(the shared scratch must not carry anything over from one call to the next).

Collected last on purpose (file name), so a failure here comes after every
other test has run; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

TOL = 1e-9   # the engine tests' tolerance for (gradient, Hessian)


def _columns(data):
    """A dense column (the intercept) and a spread of indicator columns."""
    js = [1 if data.has_offset else 0]
    ind = [j for j in range(data.J) if data.col_format[j] == 2]
    js += ind[:: max(1, len(ind) // 6)][:6]
    dense = [j for j in range(data.J) if data.col_format[j] == 0 and j not in js]
    return js + dense[:2]


@pytest.mark.parametrize("name", ["lr_laplace_small", "lr_normal_weighted", "pr_laplace_weighted"])
def test_noalloc_matches_engine_twice(cuda_lib, name):
    import torch
    from cyclops_b200 import api, _native as N
    from cyclops_b200 import data as D

    data, s = load_golden(name)
    w = s["weights"]
    use = w is not None
    eng = api.Engine(api.Dataset(data))
    eng.set_weights(w, use_cv=use)
    eng.compute_fixed_terms_in_gradient_and_hessian(use)
    eng.compute_xbeta(s["probe_beta"], use)
    eng.compute_remaining_statistics(use)
    xb = eng.get_xbeta()

    dev = torch.device("cuda:0")
    exb = np.exp(xb)
    d_exb = torch.tensor(exb, dtype=torch.float64, device=dev)
    d_den = torch.tensor(1.0 + exb, dtype=torch.float64, device=dev)
    d_w = torch.tensor(w, dtype=torch.float64, device=dev) if use else None
    d_out = torch.zeros(2, dtype=torch.float64, device=dev)
    lib = cuda_lib

    for j in _columns(data):
        g_ref, h_ref = eng.compute_gradient_and_hessian(j, use)
        rows, vals = data.column(j)
        fmt = int(data.col_format[j])
        d_rows = torch.tensor(rows, dtype=torch.int32, device=dev) if fmt in (D.SPARSE, D.INDICATOR) else None
        d_vals = torch.tensor(vals, dtype=torch.float64, device=dev) if vals is not None else None
        x = np.ones(rows.shape[0]) if vals is None else vals
        xjy = float(np.sum(x * data.y[rows] * (w[rows] if use else 1.0)))
        for call in range(2):
            d_out.fill_(np.nan)
            rc = lib.cyc_gradient_hessian_noalloc(
                int(data.model), fmt, int(rows.shape[0]),
                None if d_rows is None else d_rows.data_ptr(),
                None if d_vals is None else d_vals.data_ptr(),
                d_exb.data_ptr(), d_den.data_ptr(), None if d_w is None else d_w.data_ptr(),
                xjy, d_out.data_ptr(), C.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0, lib.cyc_last_error()
            torch.cuda.synchronize()
            g, h = d_out.cpu().numpy()
            scale = abs(h_ref) + 1.0
            assert abs(g - g_ref) <= TOL * (abs(g_ref) + scale), (name, j, call, g, g_ref)
            assert abs(h - h_ref) <= TOL * scale, (name, j, call, h, h_ref)


def test_noalloc_rejects_oversized_column(cuda_lib):
    import torch
    d = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    rc = cuda_lib.cyc_gradient_hessian_noalloc(0, 3, 4_194_305, None, None, d.data_ptr(), d.data_ptr(), None,
                                               0.0, d.data_ptr(), None)
    assert rc == 1
    assert b"4,194,304" in cuda_lib.cyc_last_error()

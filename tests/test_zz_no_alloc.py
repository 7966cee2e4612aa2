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


def _sparse_data(model, seed=3):
    """An intercept, real-valued sparse columns and indicator columns."""
    from cyclops_b200 import data as D
    rng = np.random.default_rng(seed)
    K = 6_000
    b = D.ColumnBuilder(K).intercept()
    for n in (7, 150, 900, 2_500):
        rows = np.sort(rng.choice(K, size=n, replace=False))
        b.sparse(rows, rng.normal(0.0, 1.0, size=n))
    for n in (40, 1_200):
        b.indicator(np.sort(rng.choice(K, size=n, replace=False)))
    y = (rng.random(K) < 0.3).astype(float) if model == D.LR else rng.poisson(0.7, size=K).astype(float)
    return b.build(model, y, has_intercept=True)


def _engine_state(data, beta, w):
    from cyclops_b200 import api
    use = w is not None
    eng = api.Engine(api.Dataset(data))
    eng.set_weights(w, use_cv=use)
    eng.compute_fixed_terms_in_gradient_and_hessian(use)
    eng.compute_xbeta(beta, use)
    eng.compute_remaining_statistics(use)
    return eng


@pytest.mark.parametrize("model", [0, 1])
def test_noalloc_sparse_columns(cuda_lib, model):
    """Real-valued sparse columns (row ids and values, the non-indicator
    Hessian over gathered rows) as well as indicator and dense ones, with
    row weights, against the engine; two calls per column."""
    import torch
    from cyclops_b200 import data as D
    data = _sparse_data(model)
    rng = np.random.default_rng(11)
    beta = rng.normal(0.0, 0.2, size=data.J)
    w = (rng.random(data.K) < 0.8).astype(float) * (1.0 + rng.random(data.K))
    eng = _engine_state(data, beta, w)
    xb = eng.get_xbeta()
    dev = torch.device("cuda:0")
    exb = np.exp(xb)
    d_exb = torch.tensor(exb, dtype=torch.float64, device=dev)
    d_den = torch.tensor(1.0 + exb, dtype=torch.float64, device=dev)
    d_w = torch.tensor(w, dtype=torch.float64, device=dev)
    d_out = torch.zeros(2, dtype=torch.float64, device=dev)
    assert int(np.sum(data.col_format == D.SPARSE)) == 4
    for j in range(data.J):
        g_ref, h_ref = eng.compute_gradient_and_hessian(j, True)
        rows, vals = data.column(j)
        fmt = int(data.col_format[j])
        d_rows = torch.tensor(rows, dtype=torch.int32, device=dev) if fmt in (D.SPARSE, D.INDICATOR) else None
        d_vals = torch.tensor(vals, dtype=torch.float64, device=dev) if vals is not None else None
        x = np.ones(rows.shape[0]) if vals is None else vals
        xjy = float(np.sum(x * data.y[rows] * w[rows]))
        for call in range(2):
            d_out.fill_(np.nan)
            rc = cuda_lib.cyc_gradient_hessian_noalloc(
                int(data.model), fmt, int(rows.shape[0]),
                None if d_rows is None else d_rows.data_ptr(), None if d_vals is None else d_vals.data_ptr(),
                d_exb.data_ptr(), d_den.data_ptr(), d_w.data_ptr(), xjy, d_out.data_ptr(),
                C.c_void_p(torch.cuda.current_stream().cuda_stream))
            assert rc == 0, cuda_lib.cyc_last_error()
            torch.cuda.synchronize()
            g, h = d_out.cpu().numpy()
            scale = abs(h_ref) + 1.0
            assert abs(g - g_ref) <= TOL * (abs(g_ref) + scale), (model, j, call, g, g_ref)
            assert abs(h - h_ref) <= TOL * scale, (model, j, call, h, h_ref)


def test_noalloc_takes_no_device_memory(cuda_lib):
    """After a first call (which looks up the scratch address on this device),
    further calls leave the device's free memory exactly as it was."""
    import torch
    from cyclops_b200 import data as D
    data = _sparse_data(D.LR, seed=5)
    dev = torch.device("cuda:0")
    rows, vals = data.column(3)
    d_rows = torch.tensor(rows, dtype=torch.int32, device=dev)
    d_vals = torch.tensor(vals, dtype=torch.float64, device=dev)
    d_exb = torch.ones(data.K, dtype=torch.float64, device=dev)
    d_den = torch.full((data.K,), 2.0, dtype=torch.float64, device=dev)
    d_out = torch.zeros(2, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        return cuda_lib.cyc_gradient_hessian_noalloc(0, D.SPARSE, int(rows.shape[0]), d_rows.data_ptr(),
                                                     d_vals.data_ptr(), d_exb.data_ptr(), d_den.data_ptr(), None,
                                                     0.0, d_out.data_ptr(), stream)
    assert call() == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        assert call() == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0, (free0, free1)
    g, h = d_out.cpu().numpy()
    # exp(x beta) = 1, denominators 2: the logistic terms are x/2 and x^2/4
    assert abs(g - float(np.sum(0.5 * vals))) <= 1e-12 * (1.0 + abs(g))
    assert abs(h - float(np.sum(0.25 * vals * vals))) <= 1e-12 * (1.0 + abs(h))


def test_noalloc_rejects_oversized_column(cuda_lib):
    import torch
    d = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    rc = cuda_lib.cyc_gradient_hessian_noalloc(0, 3, 4_194_305, None, None, d.data_ptr(), d.data_ptr(), None,
                                               0.0, d.data_ptr(), None)
    assert rc == 1
    assert b"4,194,304" in cuda_lib.cyc_last_error()

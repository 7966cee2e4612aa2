"""The FP64 model means of the batched solver (cyclops_b200/csrc/
fast_math.cuh: a table-driven exp after Tang, a Newton-refined reciprocal)
against an extended-precision reference and against CUDA's own exp and
division (torch on the GPU): within a few units in the last place, as exp()
followed by an IEEE division is."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = np.longdouble


def _ulps(got, want):
    want64 = want.astype(np.float64)
    return (np.abs(got.astype(L) - want) / np.spacing(np.abs(want64)).astype(L)).astype(np.float64)


def _means(lib, model, v):
    out = np.empty_like(v)
    assert lib.cyc_model_mean(model, v.size, v.ctypes.data, out.ctypes.data) == 0, lib.cyc_last_error()
    return out


def _args(rng):
    return np.concatenate([rng.uniform(-700.0, 700.0, 100_000), rng.uniform(-40.0, 40.0, 100_000),
                           rng.uniform(-1e-3, 1e-3, 20_000), np.array([0.0, -0.0, 1e-300, -1e-300, 39.99, 40.01,
                                                                       -39.99, -40.01, 707.9, -707.9, 708.5,
                                                                       -708.5, -745.5, 709.9])])


def test_exp_against_extended_precision_and_cuda(cuda_lib):
    import torch
    rng = np.random.default_rng(1)
    v = _args(rng)
    got = _means(cuda_lib, 1, v)                        # pr: exp(v)
    want = np.exp(v.astype(L))
    fin = np.isfinite(want.astype(np.float64)) & (np.abs(v) < 708.0)
    assert _ulps(got[fin], want[fin]).max() <= 1.0
    cuda = torch.exp(torch.tensor(v, dtype=torch.float64, device="cuda:0")).cpu().numpy()
    both = np.isfinite(cuda) & (cuda > 0)
    assert np.all(np.abs(got[both] - cuda[both]) <= 2 * np.spacing(cuda[both]))
    assert np.array_equal(np.isinf(got), np.isinf(cuda)) and np.array_equal(got == 0, cuda == 0)


def test_logistic_mean_against_extended_precision_and_cuda(cuda_lib):
    import torch
    rng = np.random.default_rng(2)
    v = _args(rng)
    got = _means(cuda_lib, 0, v)                        # lr: 1 / (1 + exp(-v))
    want = 1 / (1 + np.exp(-v.astype(L)))
    ok = want.astype(np.float64) > 1e-300
    assert _ulps(got[ok], want[ok]).max() <= 4.0
    t = torch.tensor(v, dtype=torch.float64, device="cuda:0")
    cuda = (1.0 / (1.0 + torch.exp(-t))).cpu().numpy()
    assert np.all(np.abs(got[ok] - cuda[ok]) <= 6 * np.spacing(cuda[ok]))
    assert np.all(got[v > 40] == 1.0) and np.all(got >= 0) and np.all(got <= 1)
    nan = _means(cuda_lib, 0, np.array([np.nan]))
    assert np.isnan(nan[0])

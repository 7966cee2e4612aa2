"""TEST INFRASTRUCTURE (oracle): an independent FP64 Newton-Raphson
maximum-likelihood fit, in NumPy, for unpenalised models on tiny dense
designs.  It shares no code or arithmetic order with the reference engine or
with the C restatement (ccd_oracle.c): it maximises the same log likelihoods
by full Newton steps on the dense design, the way glm / coxph would, so it
cross-checks the reference harness (and through it the CUDA path) on the
small designs the reference's own tests use.

The log likelihoods are the reference's (src/cyclops/engine/ModelSpecifics.h):
  lr   sum_k w_k (y_k xb_k - log(1 + exp(xb_k)))             (:998-1000, :540-568)
  pr   sum_k w_k (y_k xb_k - exp(xb_k) - log(y_k!))            (:1579-1581, :1596-1601)
  cox  Breslow ties: sum over event groups g of
       sum_{events k in g} w_k xb_k - d_g log(sum_{k at risk at g} w_k exp(xb_k)),
       d_g = sum_{events in g} w_k, risk sets within strata       (:1185-1202)
Only tests/ call it.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

LR, PR, CLR, CPR, COX = 0, 1, 2, 3, 4


def dense_design(data) -> np.ndarray:
    """K x J dense matrix of a cyclops_b200.data.CyclopsData (all formats)."""
    X = np.zeros((data.K, data.J))
    for j in range(data.J):
        rows, vals = data.column(j)
        X[rows, j] = 1.0 if vals is None else vals
    return X


def _log_factorial(y):
    return np.array([math.lgamma(v + 1.0) for v in y])


def _loglik_grad_hess(model, X, y, w, beta, offset, time, strata):
    xb = X @ beta + offset
    if model == LR:
        p = 1.0 / (1.0 + np.exp(-xb))
        ll = np.sum(w * (y * xb - np.logaddexp(0.0, xb)))
        g = X.T @ (w * (y - p))
        H = -(X.T * (w * p * (1 - p))) @ X
        return ll, g, H
    if model == PR:
        mu = np.exp(xb)
        ll = np.sum(w * (y * xb - mu - _log_factorial(y)))
        g = X.T @ (w * (y - mu))
        H = -(X.T * (w * mu)) @ X
        return ll, g, H
    # Breslow partial likelihood, risk sets within strata; conditional models
    # are one risk set per stratum (every row's time equal)
    ll = 0.0
    g = np.zeros(X.shape[1])
    H = np.zeros((X.shape[1], X.shape[1]))
    ex = w * np.exp(xb)
    for s in np.unique(strata):
        rows = np.flatnonzero(strata == s)
        ev = rows[(y[rows] > 0) & (w[rows] > 0)]
        for t in np.unique(time[ev]):
            at = ev[time[ev] == t]
            d = np.sum(w[at] * y[at])
            risk = rows[time[rows] >= t]
            S0 = np.sum(ex[risk])
            S1 = X[risk].T @ ex[risk]
            S2 = (X[risk].T * ex[risk]) @ X[risk]
            ll += np.sum(w[at] * y[at] * xb[at]) - d * np.log(S0)
            g += X[at].T @ (w[at] * y[at]) - d * S1 / S0
            H -= d * (S2 / S0 - np.outer(S1, S1) / S0 ** 2)
    return ll, g, H


def newton_fit(data, weights: Optional[np.ndarray] = None, tol: float = 1e-13, max_iter: int = 200,
               fixed: Optional[dict] = None):
    """The unpenalised MLE of `data` by Newton steps with step halving.
    Returns (beta, log_likelihood) in the data's column order; the offset
    column (when present) is held at 1 as the reference holds it, and the
    columns of `fixed` ({column: value}) at their values (a profile point)."""
    X = dense_design(data)
    K, J = X.shape
    y = np.asarray(data.y, np.float64)
    w = np.ones(K) if weights is None else np.asarray(weights, np.float64)
    free = np.ones(J, bool)
    offset = np.zeros(K)
    held = dict(fixed or {})
    if data.has_offset:
        held[0] = 1.0
    for j, v in held.items():
        free[j] = False
        offset = offset + v * X[:, j]
    Xf = X[:, free]
    time = np.zeros(K) if data.time is None else np.asarray(data.time, np.float64)
    if data.model in (CLR, CPR):
        time = np.zeros(K)
    strata = np.zeros(K, np.int64) if data.pid is None else np.asarray(data.pid, np.int64)
    model = data.model
    if model in (CLR, CPR):
        model = COX
    b = np.zeros(Xf.shape[1])
    ll, g, H = _loglik_grad_hess(model, Xf, y, w, b, offset, time, strata)
    for _ in range(max_iter):
        step = np.linalg.solve(H, -g)
        t = 1.0
        while True:
            nb = b + t * step
            nll, ng, nH = _loglik_grad_hess(model, Xf, y, w, nb, offset, time, strata)
            if nll >= ll - 1e-12 * abs(ll) or t < 1e-8:
                break
            t /= 2
        done = abs(nll - ll) <= tol * (abs(nll) + 1.0) and np.max(np.abs(nb - b)) <= 1e-10 * (1 + np.max(np.abs(nb)))
        b, ll, g, H = nb, nll, ng, nH
        if done:
            break
    beta = np.zeros(J)
    beta[free] = b
    for j, v in held.items():
        beta[j] = v
    return beta, ll

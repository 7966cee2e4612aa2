"""TEST INFRASTRUCTURE (oracle): a restatement of the reference's auto-search
cross-validation, driving the C restatement's fits.

  AutoSearchCrossValidationDriver::doCrossValidationLoop
      src/cyclops/drivers/AutoSearchCrossValidationDriver.cpp:63-160
  AbstractCrossValidationDriver::doCrossValidationStep / computePointEstimate /
  computeStDev   src/cyclops/drivers/AbstractCrossValidationDriver.cpp:131-276
  UniModalSearch::tried / step, QuadrLogFit
      src/utils/HParSearch.h:28-60, src/utils/HParSearch.cpp
  ModelData::getNormalBasedDefaultVar   src/cyclops/ModelData.cpp:680-728

Cold starts (resetCoefficients): every fold's fit starts from beta = 0.
Only tests/ use it.
"""
from __future__ import annotations

import math

import numpy as np

MAX_STEPS = 50                                   # AutoSearchCrossValidationDriver.cpp:28


class UniModalSearch:
    """The reference's one-dimensional search over a variance: multiplicative
    steps of `stdstep` until the best point is bracketed, then the argmax of
    a weighted quadratic in log(variance) (weights 1 / stdev)."""

    def __init__(self, stdstep=10.0, stop_by_y=0.01, stop_by_x=math.log(1.5), first_cut=1.0):
        self.stdstep, self.stop_by_y, self.stop_by_x, self.first_cut = stdstep, stop_by_y, stop_by_x, first_cut
        self.points = {}                       # x -> (mean, stdev)
        self.best = None

    def tried(self, x, y, sd=0.0):
        self.points[x] = (y, sd)
        if len(self.points) == 1 or y > self.points[self.best][0]:
            self.best = x

    def _fit(self):
        xs = sorted(self.points)
        pos = [self.points[x][1] for x in xs if self.points[x][1] > 0]
        zero = 100.0 / min(pos) if pos else 1.0
        X = np.array([[1.0, math.log(x), math.log(x) * math.log(x)] for x in xs])
        w = np.array([1.0 / self.points[x][1] if self.points[x][1] > 0 else zero for x in xs])
        Y = np.array([self.points[x][0] for x in xs])
        XTW = X.T * w
        return np.linalg.solve(XTW @ X, XTW @ Y)

    def step(self):
        """(continue, next x, expected value at it)"""
        xs = sorted(self.points)
        n = len(xs)
        if n == 0:
            return True, 1.0, 0.0
        if n == 1:
            x = xs[0]
            return True, (x * self.stdstep if x < self.first_cut else x / self.stdstep), 0.0
        if n == 2:
            if self.points[xs[0]][0] > self.points[xs[-1]][0]:
                return True, xs[0] / self.stdstep, 0.0
            return True, xs[-1] * self.stdstep, 0.0
        b = self.best
        if xs[0] == b:
            return (b > 5e-324), b / self.stdstep, (0.0 if b > 5e-324 else self.points[b][0])
        if xs[-1] == b:
            return (b < math.inf), b * self.stdstep, (0.0 if b < math.inf else self.points[b][0])
        c0, c1, c2 = self._fit()
        log_argmax = -c1 / c2 / 2
        expected = -c1 * c1 / c2 / 4 + c0
        maxval = self.points[b][0]
        go = True
        if maxval == 0:
            go = False
        elif (expected - maxval) / abs(maxval) < self.stop_by_y:
            go = False
        elif abs(log_argmax - math.log(b)) < self.stop_by_x:
            go = False
        return go, math.exp(log_argmax), expected


def normal_based_default_variance(data) -> float:
    """sum over the variable columns of sum x^2, / their count / K (the
    intercept and offset columns, at the front, left out)."""
    start = int(data.has_intercept) + int(data.has_offset)
    total = 0.0
    for j in range(start, data.J):
        rows, vals = data.column(j)
        total += float(rows.size) if vals is None else float(np.dot(vals, vals))
    return total / (data.J - start) / data.K


def auto_search(data, fits, n_folds, fold_weights, starting_variance=-1.0):
    """fits(variance, train_weights, held_weights) -> held-out predictive log
    likelihood (NaN when the fit did not converge); fold_weights: the
    (reps * n_folds, K) training masks in the selector's order.  Returns
    (best variance, its expected value, [(variance, mean, stdev), ...])."""
    x = starting_variance if starting_variance > 0 else normal_based_default_variance(data)
    search = UniModalSearch(10.0, 0.01, math.log(1.5))
    trail = []
    value = 0.0
    for step in range(MAX_STEPS):
        pll = []
        for w in fold_weights:
            pll.append(fits(x, w, 1.0 - w))
        ok = [v for v in pll if v == v]                 # NaN (no convergence) left out
        total = 0.0
        for v in ok:
            total += v
        mean = total / len(ok)
        inner = 0.0
        for v in ok:
            inner += v * v
        sd = math.sqrt(inner / len(ok) - mean * mean)
        trail.append((x, mean, sd))
        search.tried(x, mean, sd)
        go, nx, expected = search.step()
        x, value = nx, expected
        if not go:
            break
    return x, value, trail

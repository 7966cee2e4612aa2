"""Auto-search cross-validation on the CPU: the restatement (oracle/cv_auto.py
over the C restatement's fits) against the reference's own
AutoSearchCrossValidationDriver (fixtures tests/golden/cvauto_*.npz), and
the library's C++ variance search (cyclops_b200/csrc/variance_search.h)
replaying the reference's trails point by point."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, cvauto_names, load_golden
from cyclops_b200 import data as D
from oracle import cv_auto
from oracle import oracle as O


def _fold_weights(data, by_row, seed):
    if by_row:
        ids = np.arange(data.K, dtype=np.int32)
    else:                                   # strata renumbered by runs, as the selector sees them
        pid = np.asarray(data.pid)
        ids = np.concatenate([[0], np.cumsum(pid[1:] != pid[:-1])]).astype(np.int32)
    return O.ref_cv_weights(data.K, ids, 10, seed, by_row=by_row, n_reps=1)


@pytest.mark.parametrize("name", cvauto_names())
def test_restated_auto_search_matches_reference(name):
    z = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
    data, _ = load_golden(str(z["base"]))
    prior = int(z["prior"])
    W = _fold_weights(data, bool(z["by_row"]), int(z["seed"]))

    def fits(v, w, held):
        f = O.port().fit(data, prior, v, weights=w)
        return float("nan") if f.return_flag != 0 else O.port().predictive_loglik(data, f.beta, held)

    x, value, trail = cv_auto.auto_search(data, fits, 10, W, float(z["starting_variance"]))
    np.testing.assert_allclose(x, float(z["best_variance"]), rtol=1e-9)
    np.testing.assert_allclose(value, float(z["best_value"]), rtol=1e-9)
    np.testing.assert_allclose(np.array(trail), z["tried"], rtol=1e-5)      # the driver logs 6 digits


_REPLAY = r"""
#include <cstdio>
#include "variance_search.h"
int main() {
    cyc::VarianceSearch s;
    double x, m, sd;
    while (std::scanf("%lf %lf %lf", &x, &m, &sd) == 3) {
        s.tried(x, m, sd);
        bool go; double nx, e;
        s.step(&go, &nx, &e);
        std::printf("%d %.17g %.17g\n", go ? 1 : 0, nx, e);
    }
    return 0;
}
"""


def test_library_variance_search_replays_reference_trails(tmp_path):
    """Fed the restatement's full-precision trail of each case, the C++
    search proposes the same next point after every step and stops where
    the reference stopped, on the variance the reference chose."""
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "replay.cpp"
    src.write_text(_REPLAY)
    exe = tmp_path / "replay"
    subprocess.run([cxx, "-std=c++14", "-O2", "-I", os.path.join(ROOT, "cyclops_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    for name in cvauto_names():
        z = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
        data, _ = load_golden(str(z["base"]))
        prior = int(z["prior"])
        W = _fold_weights(data, bool(z["by_row"]), int(z["seed"]))

        def fits(v, w, held):
            f = O.port().fit(data, prior, v, weights=w)
            return float("nan") if f.return_flag != 0 else O.port().predictive_loglik(data, f.beta, held)

        x, value, trail = cv_auto.auto_search(data, fits, 10, W, float(z["starting_variance"]))
        feed = "\n".join(f"{a!r} {b!r} {c!r}" for a, b, c in trail)
        out = subprocess.run([str(exe)], input=feed, capture_output=True, text=True, check=True).stdout.split("\n")
        steps = [l.split() for l in out if l.strip()]
        for i, (go, nx, e) in enumerate(steps[:-1]):
            assert go == "1"
            np.testing.assert_allclose(float(nx), trail[i + 1][0], rtol=1e-12)
        go, nx, e = steps[-1]
        assert go == "0" or len(steps) == cv_auto.MAX_STEPS
        np.testing.assert_allclose(float(nx), float(z["best_variance"]), rtol=1e-9)
        np.testing.assert_allclose(float(e), float(z["best_value"]), rtol=1e-9)


@pytest.mark.parametrize("name,weighted", [("lr_laplace_small", True), ("lr_laplace_small", False),
                                           ("cpr_normal", True), ("cox_laplace", False), ("cox_strata", True)])
def test_restated_grid_cv_matches_reference_driver(name, weighted):
    """The reference's GridSearchCrossValidationDriver (cold starts), with
    the fit's observation weights as the selector's original weights: each
    fold trains at the weights outside it and is scored at the weights
    inside it (getComplement) -- the semantics cyc_cv_grid_fit_weighted
    implements -- reproduced fold by fold by the restatement.  Cox folds
    are by row (R's "auto" selector picks byRow when a stratum holds at
    least as many rows as there are strata, R/ModelFit.R:174-184), and a
    held-out fold is scored against the risk sets of the training rows."""
    data, s = load_golden(name)
    prior = int(s["prior"])
    by_row = data.pid is None or data.model == D.COX
    w = (1.0 + (np.arange(data.K) % 3)) if weighted else None
    pts, vals, fp = O.ref().cv_grid(data, prior, fold=5, seed=77, by_row=by_row, lower=0.05, upper=5.0,
                                    grid_steps=3, weights=w)
    if by_row:
        ids = np.arange(data.K, dtype=np.int32)
    else:
        pid = np.asarray(data.pid)
        ids = np.concatenate([[0], np.cumsum(pid[1:] != pid[:-1])]).astype(np.int32)
    masks = O.ref_cv_weights(data.K, ids, 5, 77, by_row=by_row, n_reps=1)
    base = np.ones(data.K) if w is None else w
    for g, v in enumerate(pts):
        got = []
        for f in range(5):
            train = masks[f] * base
            held = (1.0 - masks[f]) * base
            fit = O.port().fit(data, prior, v, weights=train)
            got.append(O.port().predictive_loglik(data, fit.beta, held, weights=train)
                       if fit.return_flag == 0 else float("nan"))
        np.testing.assert_allclose(got, fp[g], rtol=1e-5)
        np.testing.assert_allclose(np.nanmean(got), vals[g], rtol=1e-9)

"""Host-side data container and seeded synthetic generators.

`CyclopsData` is the column store the CUDA engine ingests: the same column
order, formats and row order as the reference's `ModelData` after R's
`createCyclopsData` (reference: src/RcppModelData.cpp:751-900,
R/DataManagement.R:158-176):

* column 0 is the fixed offset (beta = 1) when ``has_offset``;
* then dense columns (the intercept first), then sparse, then indicator;
* survival rows are sorted by (stratum, -time, y); stratified non-survival
  rows by stratum; stratum ids are renumbered 0..S-1 by runs
  (src/RcppModelData.cpp:878-900).

Formats follow `FormatType` (src/cyclops/CompressedDataMatrix.h:36-38):
DENSE=0, SPARSE=1, INDICATOR=2, INTERCEPT=3.  Row ids inside a column are
ascending int32; SPARSE values are float64 parallel to them; DENSE columns
hold K float64 values.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence

import numpy as np

DENSE, SPARSE, INDICATOR, INTERCEPT = 0, 1, 2, 3
LR, PR, CLR, CPR, COX = 0, 1, 2, 3, 4
MODEL_NAMES = {"lr": LR, "pr": PR, "clr": CLR, "cpr": CPR, "cox": COX}
PRIOR_NONE, PRIOR_LAPLACE, PRIOR_NORMAL = 0, 1, 2
CONV_GRADIENT, CONV_LANGE, CONV_MITTAL, CONV_ONE_STEP, CONV_ZHANG_OLES = range(5)


@dataclasses.dataclass
class CyclopsData:
    model: int
    y: np.ndarray                      # (K,) float64
    col_format: np.ndarray             # (J,) int32
    col_ptr: np.ndarray                # (J+1,) int64 into col_idx
    col_idx: np.ndarray                # int32 row ids
    val_ptr: np.ndarray                # (J+1,) int64 into col_val
    col_val: np.ndarray                # float64
    pid: Optional[np.ndarray] = None   # (K,) int32 raw stratum ids (renumbered by runs)
    time: Optional[np.ndarray] = None  # (K,) float64 survival times
    has_offset: bool = False
    has_intercept: bool = False

    @property
    def K(self) -> int:
        return int(self.y.shape[0])

    @property
    def J(self) -> int:
        return int(self.col_format.shape[0])

    @property
    def nnz(self) -> int:
        return int(self.col_idx.shape[0])

    def column(self, j: int):
        """(rows, values) of column j as arrays (values None for indicators)."""
        f = int(self.col_format[j])
        if f in (DENSE, INTERCEPT):
            rows = np.arange(self.K, dtype=np.int32)
        else:
            rows = self.col_idx[self.col_ptr[j]:self.col_ptr[j + 1]]
        if f in (DENSE, SPARSE):
            n = self.K if f == DENSE else rows.shape[0]
            vals = self.col_val[self.val_ptr[j]:self.val_ptr[j] + n]
        else:
            vals = None
        return rows, vals

    def dense_matrix(self) -> np.ndarray:
        """K x J dense float64 copy (small problems only)."""
        X = np.zeros((self.K, self.J))
        for j in range(self.J):
            rows, vals = self.column(j)
            X[rows, j] = 1.0 if vals is None else vals
        return X

    def strata(self) -> np.ndarray:
        """Stratum of each row renumbered by runs (RcppModelData.cpp:878-900)."""
        if self.pid is None:
            return np.arange(self.K, dtype=np.int32)
        p = np.asarray(self.pid)
        change = np.empty(self.K, dtype=np.int32)
        change[0] = 0
        change[1:] = (p[1:] != p[:-1])
        return np.cumsum(change, dtype=np.int64).astype(np.int32)

    def validate(self) -> None:
        K, J = self.K, self.J
        if self.col_ptr.shape != (J + 1,) or self.val_ptr.shape != (J + 1,):
            raise ValueError("col_ptr/val_ptr must have J+1 entries")
        for j in range(J):
            f = int(self.col_format[j])
            n_idx = int(self.col_ptr[j + 1] - self.col_ptr[j])
            n_val = int(self.val_ptr[j + 1] - self.val_ptr[j])
            if f == DENSE and (n_idx != 0 or n_val != K):
                raise ValueError(f"dense column {j} must hold K values")
            if f == SPARSE and n_val != n_idx:
                raise ValueError(f"sparse column {j}: values/indices mismatch")
            if f in (INDICATOR, INTERCEPT) and n_val != 0:
                raise ValueError(f"column {j} must hold no values")
            if f == INTERCEPT and n_idx != 0:
                raise ValueError(f"intercept column {j} must hold no indices")
        if self.nnz:
            if self.col_idx.min() < 0 or self.col_idx.max() >= K:
                raise ValueError("row index out of range")
        for j in range(J):
            r = self.col_idx[self.col_ptr[j]:self.col_ptr[j + 1]]
            if r.shape[0] > 1 and np.any(np.diff(r) <= 0):
                raise ValueError(f"column {j}: row ids must be strictly ascending")
        if self.model == COX and self.time is None:
            raise ValueError("cox needs survival times")


class ColumnBuilder:
    """Accumulates columns in reference ingest order."""

    def __init__(self, K: int):
        self.K = K
        self.fmt: list[int] = []
        self.idx: list[np.ndarray] = []
        self.val: list[np.ndarray] = []

    def dense(self, values) -> "ColumnBuilder":
        v = np.ascontiguousarray(values, dtype=np.float64)
        assert v.shape == (self.K,)
        self.fmt.append(DENSE)
        self.idx.append(np.zeros(0, np.int32))
        self.val.append(v)
        return self

    def intercept(self, as_dense: bool = True) -> "ColumnBuilder":
        if as_dense:
            return self.dense(np.ones(self.K))
        self.fmt.append(INTERCEPT)
        self.idx.append(np.zeros(0, np.int32))
        self.val.append(np.zeros(0))
        return self

    def sparse(self, rows, values) -> "ColumnBuilder":
        rows = np.asarray(rows, dtype=np.int32)
        values = np.asarray(values, dtype=np.float64)
        o = np.argsort(rows, kind="stable")
        self.fmt.append(SPARSE)
        self.idx.append(rows[o])
        self.val.append(values[o])
        return self

    def indicator(self, rows) -> "ColumnBuilder":
        rows = np.sort(np.asarray(rows, dtype=np.int32))
        self.fmt.append(INDICATOR)
        self.idx.append(rows)
        self.val.append(np.zeros(0))
        return self

    def indicator_csc(self, indptr: np.ndarray, indices: np.ndarray) -> "ColumnBuilder":
        """Append many indicator columns at once from CSC arrays (rows sorted per column)."""
        n = indptr.shape[0] - 1
        for c in range(n):
            self.fmt.append(INDICATOR)
            self.idx.append(indices[indptr[c]:indptr[c + 1]])
            self.val.append(np.zeros(0))
        return self

    def build(self, model: int, y, pid=None, time=None, has_offset=False,
              has_intercept=False) -> CyclopsData:
        fmt = np.asarray(self.fmt, dtype=np.int32)
        col_ptr = np.zeros(len(fmt) + 1, np.int64)
        val_ptr = np.zeros(len(fmt) + 1, np.int64)
        col_ptr[1:] = np.cumsum([a.shape[0] for a in self.idx])
        val_ptr[1:] = np.cumsum([a.shape[0] for a in self.val])
        idx = np.concatenate(self.idx) if self.idx else np.zeros(0, np.int32)
        val = np.concatenate(self.val) if self.val else np.zeros(0)
        return CyclopsData(
            model=model, y=np.ascontiguousarray(y, dtype=np.float64), col_format=fmt,
            col_ptr=col_ptr, col_idx=np.ascontiguousarray(idx, dtype=np.int32),
            val_ptr=val_ptr, col_val=np.ascontiguousarray(val, dtype=np.float64),
            pid=None if pid is None else np.ascontiguousarray(pid, dtype=np.int32),
            time=None if time is None else np.ascontiguousarray(time, dtype=np.float64),
            has_offset=has_offset, has_intercept=has_intercept)


# --------------------------------------------------------------------------
# seeded synthetic generators (numpy PCG64)
# --------------------------------------------------------------------------

def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _bernoulli_csc(rng, K: int, P: int, density: float):
    """CSC of a K x P 0/1 matrix with i.i.d. Bernoulli(density) entries."""
    counts = rng.binomial(K, density, size=P)
    indptr = np.zeros(P + 1, np.int64)
    indptr[1:] = np.cumsum(counts)
    indices = np.empty(int(indptr[-1]), np.int32)
    for c in range(P):
        n = int(counts[c])
        if n:
            indices[indptr[c]:indptr[c + 1]] = np.sort(rng.choice(K, size=n, replace=False))
    return indptr, indices


def _zipf_column_counts(rng, K: int, P: int, total: int, s: float):
    """Column sizes proportional to rank^-s, capped at K, scaled so that the
    capped sizes still add up to `total` (bisection on the scale)."""
    w = np.arange(1, P + 1, dtype=np.float64) ** (-s)
    w /= w.sum()
    lo, hi = 1.0, 1.0
    while np.minimum(w * total * hi, K).sum() < total and hi < 1e6:
        hi *= 2.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if np.minimum(w * total * mid, K).sum() < total:
            lo = mid
        else:
            hi = mid
    n = np.minimum(np.floor(w * total * hi + rng.random(P)).astype(np.int64), K)
    return n


def _csc_from_counts(rng, K: int, counts: np.ndarray):
    P = counts.shape[0]
    indptr = np.zeros(P + 1, np.int64)
    indptr[1:] = np.cumsum(counts)
    indices = np.empty(int(indptr[-1]), np.int32)
    for c in range(P):
        n = int(counts[c])
        if n == 0:
            continue
        if n > K // 4:
            rows = np.sort(rng.choice(K, size=n, replace=False)).astype(np.int32)
        else:
            rows = np.unique(rng.integers(0, K, size=int(n * 1.1) + 8).astype(np.int32))
            if rows.shape[0] > n:
                rows = np.sort(rng.choice(rows, size=n, replace=False))
        counts[c] = rows.shape[0]
        indices[indptr[c]:indptr[c] + rows.shape[0]] = rows
    # re-pack if some columns came out shorter than requested
    new_ptr = np.zeros(P + 1, np.int64)
    new_ptr[1:] = np.cumsum(counts)
    if new_ptr[-1] != indptr[-1]:
        packed = np.empty(int(new_ptr[-1]), np.int32)
        for c in range(P):
            packed[new_ptr[c]:new_ptr[c + 1]] = indices[indptr[c]:indptr[c] + counts[c]]
        indices, indptr = packed, new_ptr
    return indptr, indices


def _csc_matvec(indptr, indices, beta_cols: np.ndarray, K: int) -> np.ndarray:
    """x = X @ beta for an indicator CSC matrix, only over nonzero beta."""
    out = np.zeros(K)
    for c in np.flatnonzero(beta_cols):
        out[indices[indptr[c]:indptr[c + 1]]] += beta_cols[c]
    return out


def synth_logistic(K=10_000, P=1_000, density=0.01, n_true=50, sd_true=0.5,
                   intercept=-2.0, seed=1, zipf: Optional[float] = None) -> CyclopsData:
    """Logistic regression with a dense intercept and P indicator columns.

    Uniform density (zipf=None) is the 10k x 1k, 1 % workload; with ``zipf``
    column frequencies follow Zipf(zipf) at the given mean density (the
    500k x 20k, 0.2 % cross-validation workload)."""
    rng = _rng(seed)
    if zipf is None:
        indptr, indices = _bernoulli_csc(rng, K, P, density)
    else:
        counts = _zipf_column_counts(rng, K, P, int(round(density * K * P)), zipf)
        indptr, indices = _csc_from_counts(rng, K, counts)
    beta = np.zeros(P)
    cols = rng.choice(P, size=min(n_true, P), replace=False)
    beta[cols] = rng.normal(0.0, sd_true, size=cols.shape[0])
    eta = intercept + _csc_matvec(indptr, indices, beta, K)
    y = (rng.random(K) < 1.0 / (1.0 + np.exp(-eta))).astype(np.float64)
    b = ColumnBuilder(K).intercept().indicator_csc(indptr, indices)
    return b.build(LR, y, has_intercept=True)


def _zipf_rows_without_replacement(rng, K: int, P: int, per_row: int, s: float,
                                   chunk: int = 65536):
    """Each row draws `per_row` distinct columns with probability ~ rank^-s.

    Draws with replacement and keeps the first `per_row` distinct ones, which
    is successive sampling without replacement proportional to the weights."""
    w = np.arange(1, P + 1, dtype=np.float64) ** (-s)
    cdf = np.cumsum(w / w.sum())
    cdf[-1] = 1.0
    rows_out, cols_out = [], []
    m = per_row * 3
    for r0 in range(0, K, chunk):
        r1 = min(K, r0 + chunk)
        n = r1 - r0
        draws = np.searchsorted(cdf, rng.random((n, m))).astype(np.int32)
        order = np.argsort(draws, axis=1, kind="stable")
        sd = np.take_along_axis(draws, order, axis=1)
        first = np.ones_like(sd, dtype=bool)
        first[:, 1:] = sd[:, 1:] != sd[:, :-1]
        keep_sorted = np.zeros_like(first)
        np.put_along_axis(keep_sorted, order, first, axis=1)   # first occurrences, draw order
        rank = np.cumsum(keep_sorted, axis=1)
        sel = keep_sorted & (rank <= per_row)
        rr, cc = np.nonzero(sel)
        rows_out.append((rr + r0).astype(np.int32))
        cols_out.append(draws[rr, cc])
    rows = np.concatenate(rows_out)
    cols = np.concatenate(cols_out)
    order = np.lexsort((rows, cols))
    rows, cols = rows[order], cols[order]
    indptr = np.zeros(P + 1, np.int64)
    indptr[1:] = np.cumsum(np.bincount(cols, minlength=P))
    return indptr, rows


def synth_poisson(K=1_000_000, P=100_000, per_row=50, zipf=1.1, n_dense=10, n_true=500,
                  sd_true=0.3, intercept=-1.0, seed=2, offset=True) -> CyclopsData:
    """Poisson regression: offset log(t), t ~ Exp(1) (fixed column 0), an
    intercept, `n_dense` N(0,1) dense columns and P indicator columns with
    `per_row` distinct Zipf(zipf)-ranked columns per row."""
    rng = _rng(seed)
    t = rng.exponential(1.0, size=K)
    dense = rng.normal(0.0, 1.0, size=(n_dense, K))
    indptr, indices = _zipf_rows_without_replacement(rng, K, P, per_row, zipf)
    beta = np.zeros(P + n_dense)
    cols = rng.choice(P + n_dense, size=min(n_true, P + n_dense), replace=False)
    beta[cols] = rng.normal(0.0, sd_true, size=cols.shape[0])
    eta = intercept + dense.T @ beta[:n_dense] + _csc_matvec(indptr, indices, beta[n_dense:], K)
    if offset:
        eta = eta + np.log(t)
    y = rng.poisson(np.exp(np.minimum(eta, 30.0))).astype(np.float64)
    b = ColumnBuilder(K)
    if offset:
        b.dense(np.log(t))
    b.intercept()
    for d in range(n_dense):
        b.dense(dense[d])
    b.indicator_csc(indptr, indices)
    return b.build(PR, y, time=np.log(t) if offset else None, has_offset=offset,
                   has_intercept=True)


def synth_cox(K=2_000_000, P=50_000, density=0.0005, shape=1.2, scale=1.0, censor=0.7,
              n_strata=0, n_true=100, sd_true=0.3, seed=3, ties: Optional[int] = None,
              indicator=False) -> CyclopsData:
    """Breslow Cox: Weibull(shape, scale) proportional-hazards times, random
    censoring, P sparse N(0,1) columns (or indicators); rows sorted by
    (stratum, -time, y) as R does for survival models
    (R/DataManagement.R:164-172).  ``ties`` rounds times to that many
    decimals to create tied event times."""
    rng = _rng(seed)
    indptr, indices = _bernoulli_csc(rng, K, P, density)
    vals = rng.normal(0.0, 1.0, size=indices.shape[0])
    beta = np.zeros(P)
    cols = rng.choice(P, size=min(n_true, P), replace=False)
    beta[cols] = rng.normal(0.0, sd_true, size=cols.shape[0])
    eta = np.zeros(K)
    for c in cols:
        sl = slice(indptr[c], indptr[c + 1])
        eta[indices[sl]] += beta[c] * (1.0 if indicator else vals[sl])
    e = rng.exponential(1.0, size=K)
    time = scale * (e / np.exp(eta)) ** (1.0 / shape)
    if ties is not None:
        time = np.round(time, ties) + 10.0 ** (-ties)
    y = (rng.random(K) >= censor).astype(np.float64)
    strata = rng.integers(0, n_strata, size=K) if n_strata else np.zeros(K, np.int64)
    order = np.lexsort((y, -time, strata))            # order(pid, -time, y)
    inv = np.empty(K, np.int64)
    inv[order] = np.arange(K)
    y, time, strata = y[order], time[order], strata[order]
    b = ColumnBuilder(K)
    col_vals = np.ones_like(vals) if indicator else vals
    for c in range(P):
        sl = slice(indptr[c], indptr[c + 1])
        rows = inv[indices[sl]]
        if indicator:
            b.indicator(rows)
        else:
            b.sparse(rows, col_vals[sl])
    return b.build(COX, y, pid=strata.astype(np.int32), time=time)


def synth_conditional(K=20_000, P=500, density=0.01, stratum_size=5, n_true=30,
                      sd_true=0.5, seed=4, model=CLR) -> CyclopsData:
    """Matched strata (1:(stratum_size-1) for clr), P indicator columns.
    Rows are sorted by stratum (R/DataManagement.R:168)."""
    rng = _rng(seed)
    S = K // stratum_size
    K = S * stratum_size
    indptr, indices = _bernoulli_csc(rng, K, P, density)
    beta = np.zeros(P)
    cols = rng.choice(P, size=min(n_true, P), replace=False)
    beta[cols] = rng.normal(0.0, sd_true, size=cols.shape[0])
    eta = _csc_matvec(indptr, indices, beta, K)
    pid = np.repeat(np.arange(S, dtype=np.int32), stratum_size)
    if model == CLR:
        # one case per stratum, chosen with probability softmax(eta)
        p = np.exp(eta).reshape(S, stratum_size)
        p /= p.sum(axis=1, keepdims=True)
        u = rng.random(S)[:, None]
        case = (np.cumsum(p, axis=1) < u).sum(axis=1)
        y = np.zeros((S, stratum_size))
        y[np.arange(S), np.minimum(case, stratum_size - 1)] = 1.0
        y = y.reshape(K)
    else:
        y = rng.poisson(np.exp(eta)).astype(np.float64)
    b = ColumnBuilder(K).indicator_csc(indptr, indices)
    return b.build(model, y, pid=pid)


def cv_fold_weights(K: int, folds: int, seed: int, n_reps: int = 1) -> np.ndarray:
    """0/1 row masks for `folds`-fold cross-validation by row, following the
    interval rule of CrossValidationSelector (reference:
    src/cyclops/drivers/CrossValidationSelector.cpp:31-42, 72-116): a
    seeded permutation of the rows is cut into `folds` intervals whose sizes
    differ by at most one; fold f holds out interval f.

    The permutation here comes from numpy's PCG64 generator; the reference
    uses std::mt19937 + std::shuffle, so individual masks differ while the
    interval sizes match exactly."""
    rng = _rng(seed)
    starts = [0]
    frac, extra = K // folds, K - (K // folds) * folds
    for i in range(folds):
        starts.append(starts[-1] + frac + (1 if i < extra else 0))
    out = np.ones((n_reps * folds, K))
    for r in range(n_reps):
        perm = rng.permutation(K)
        for f in range(folds):
            out[r * folds + f, perm[starts[f]:starts[f + 1]]] = 0.0
    return out


def lambda_grid(lo: float, hi: float, n: int) -> np.ndarray:
    """Log-uniform grid (GridSearchCrossValidationDriver.cpp:38-48)."""
    if n == 1:
        return np.array([hi])
    step = (math.log(hi) - math.log(lo)) / (n - 1)
    return np.exp(math.log(lo) + step * np.arange(n))


def laplace_variance(lam: float) -> float:
    """Cyclops takes a prior variance; Laplace rate lambda = sqrt(2/variance)
    (src/cyclops/priors/CovariatePrior.h:282-292)."""
    return 2.0 / (lam * lam)

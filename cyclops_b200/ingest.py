"""Ingest: outcome and covariate tables in long format (the Andromeda / SQL
layout: one row per (rowId, covariateId, covariateValue)) into the column
store the engine reads, by the reference's rules, so that row order, column
order, column formats and strata come out exactly as the reference's.

Two halves, as in the reference:

* sorting (the R layer, convertToCyclopsData, R/NewDataConversion.R:94-176):
  lr / pr outcomes by rowId and covariates by (covariateId, rowId); clr / cpr
  outcomes by (stratumId, rowId) and covariates by (covariateId, stratumId,
  rowId); cox outcomes by (stratumId, time descending, y, rowId) and
  covariates, joined to their outcome row, by (covariateId, stratumId, time
  descending, y, rowId); stable, like R's order(); covariate rows whose rowId
  has no outcome are dropped; conditional models get no intercept;
* loading (ModelData, src/cyclops/ModelData.cpp): loadY maps each rowId to
  its position and renumbers strata by runs (:69-145); the intercept is an
  INTERCEPT column moved to the front (loadX, :246-370); loadMultipleX makes
  one column per covariateId run (:148-243): INDICATOR unless a value is
  neither 0 nor 1 (then SPARSE, earlier entries valued 1), zero values not
  stored, a repeated (row, covariate) an error; Poisson models put log(time)
  in front as the fixed offset column (setOffsetCovariate(-1) +
  logTransformCovariate(0), :609-651, via .cyclopsFinalizeData,
  src/RcppModelData.cpp:463-545).

Host-side numpy; the result uploads with `api.Dataset` like any CyclopsData.
"""
from __future__ import annotations

import math
from typing import Mapping, Optional, Tuple

import numpy as np

from . import data as D

_MODELS = {"lr": D.LR, "pr": D.PR, "clr": D.CLR, "cpr": D.CPR, "cox": D.COX}


class IngestError(ValueError):
    pass


def _col(t: Mapping, name: str, dtype=None):
    if name not in t or t[name] is None:
        return None
    a = np.asarray(t[name])
    return a.astype(dtype) if dtype is not None else a


def _stable_order(*keys):
    """R's order(k0, k1, ...): the first key is primary; ties keep input order."""
    return np.lexsort(tuple(reversed(keys)))


def sort_outcomes(model: int, outcomes: Mapping) -> dict:
    """The R layer's outcome sort (R/NewDataConversion.R:125-160)."""
    row = _col(outcomes, "rowId", np.int64)
    y = _col(outcomes, "y", np.float64)
    if row is None or y is None:
        raise IngestError("outcomes need rowId and y")
    stratum = _col(outcomes, "stratumId", np.int64)
    time = _col(outcomes, "time", np.float64)
    weights = _col(outcomes, "weights", np.float64)
    if model in (D.LR, D.PR):
        stratum = None
        o = _stable_order(row)
    elif model in (D.CLR, D.CPR):
        if stratum is None:
            raise IngestError("conditional models need outcomes$stratumId")
        o = _stable_order(stratum, row)
    else:
        if time is None:
            raise IngestError("cox needs outcomes$time")
        if np.unique(y).size > 2:
            raise IngestError("Cox model only accepts one outcome type")
        if stratum is None:
            stratum = np.zeros(row.size, np.int64)
        o = _stable_order(stratum, -time, y, row)
    pick = lambda a: None if a is None else a[o]
    return {"rowId": row[o], "y": y[o], "stratumId": pick(stratum), "time": pick(time), "weights": pick(weights)}


def sort_covariates(model: int, covariates: Mapping, outcomes_sorted: Mapping) -> dict:
    """The R layer's covariate sort, after dropping rows without an outcome
    (R/NewDataConversion.R:131-176)."""
    cid = _col(covariates, "covariateId", np.int64)
    row = _col(covariates, "rowId", np.int64)
    if cid is None or row is None:
        raise IngestError("covariates need covariateId and rowId")
    val = _col(covariates, "covariateValue", np.float64)
    orow = outcomes_sorted["rowId"]
    # position of each covariate row's outcome (the last one if a rowId repeats,
    # as the reference's rowIdMap keeps the last assignment)
    uniq, last = np.unique(orow[::-1], return_index=True)
    last = orow.size - 1 - last
    at = np.searchsorted(uniq, row)
    found = (at < uniq.size) & (uniq[np.minimum(at, uniq.size - 1)] == row)
    keep = np.flatnonzero(found)
    cid, row = cid[keep], row[keep]
    val = None if val is None else val[keep]
    pos = last[at[keep]]
    if model in (D.LR, D.PR):
        o = _stable_order(cid, row)
    elif model in (D.CLR, D.CPR):
        st = _col(covariates, "stratumId", np.int64)
        st = outcomes_sorted["stratumId"][pos] if st is None else st[keep]
        o = _stable_order(cid, st, row)
    else:
        st = outcomes_sorted["stratumId"][pos]
        tm = outcomes_sorted["time"][pos]
        yy = outcomes_sorted["y"][pos]
        o = _stable_order(cid, st, -tm, yy, row)
    return {"covariateId": cid[o], "rowId": row[o], "covariateValue": None if val is None else val[o],
            "position": pos[o]}


def load(model: int, outs: dict, covs: dict, add_intercept: bool) -> D.CyclopsData:
    """ModelData::loadY + loadX(intercept) + loadMultipleX + the Poisson
    offset, on tables already in the reference's order."""
    K = outs["rowId"].size
    # loadY: strata renumbered by runs (:100-122)
    pid = None
    if outs["stratumId"] is not None:
        s = outs["stratumId"]
        pid = np.concatenate([[0], np.cumsum(s[1:] != s[:-1])]).astype(np.int32) if K else np.zeros(0, np.int32)
    fmts, ptr, vptr, idx_parts, val_parts, labels = [], [0], [0], [], [], []

    def add(fmt, rows, vals, label):
        fmts.append(fmt)
        labels.append(label)
        if rows is not None:
            idx_parts.append(rows.astype(np.int32))
            ptr.append(ptr[-1] + rows.size)
        else:
            ptr.append(ptr[-1])
        if vals is not None:
            val_parts.append(vals.astype(np.float64))
            vptr.append(vptr[-1] + vals.size)
        else:
            vptr.append(vptr[-1])

    offset = model in (D.PR, D.CPR)
    if offset:
        t = outs["time"]
        if t is None:
            raise IngestError("Poisson models need outcomes$time")
        # setOffsetCovariate(-1) + logTransformCovariate(0): the C library log, as std::log
        add(D.DENSE, None, np.fromiter(map(math.log, t.tolist()), np.float64, t.size), -1)
    has_intercept = add_intercept and model in (D.LR, D.PR)
    if has_intercept:
        add(D.INTERCEPT, None, None, 0)                # loadX(0, none, none): INTERCEPT, to the front
    cid, pos, val = covs["covariateId"], covs["position"], covs["covariateValue"]
    if cid.size:
        starts = np.flatnonzero(np.concatenate([[True], cid[1:] != cid[:-1]]))
        ends = np.concatenate([starts[1:], [cid.size]])
        rows_all = covs["rowId"]
        # a repeated (row, covariate) entry is an error (:188-194)
        rep = (cid[1:] == cid[:-1]) & (rows_all[1:] == rows_all[:-1])
        if rep.any():
            i = int(np.flatnonzero(rep)[0]) + 1
            raise IngestError(f"Repeated row-column entry at {rows_all[i]} - {cid[i]}")
        if val is None:
            for a, b in zip(starts, ends):
                add(D.INDICATOR, pos[a:b], None, int(cid[a]))
        else:
            nz = val != 0.0
            not01 = ~((val == 0.0) | (val == 1.0))
            for a, b in zip(starts, ends):
                keep = nz[a:b]
                sparse = bool(not01[a:b].any())      # first value, or an upcast (:176-184)
                rows = pos[a:b][keep]
                add(D.SPARSE if sparse else D.INDICATOR, rows, val[a:b][keep] if sparse else None, int(cid[a]))
    col_idx = np.concatenate(idx_parts) if idx_parts else np.zeros(0, np.int32)
    col_val = np.concatenate(val_parts) if val_parts else np.zeros(0)
    cd = D.CyclopsData(model=model, y=np.ascontiguousarray(outs["y"]), col_format=np.asarray(fmts, np.int32),
                       col_ptr=np.asarray(ptr, np.int64), col_idx=np.ascontiguousarray(col_idx, np.int32),
                       val_ptr=np.asarray(vptr, np.int64), col_val=np.ascontiguousarray(col_val),
                       pid=pid, time=outs["time"], has_offset=offset, has_intercept=has_intercept)
    cd.labels = np.asarray(labels, np.int64)
    return cd


def convert_to_cyclops_data(outcomes: Mapping, covariates: Mapping, model_type: str = "lr",
                            add_intercept: bool = True) -> Tuple[D.CyclopsData, Optional[np.ndarray]]:
    """convertToCyclopsData (R/NewDataConversion.R:94-210) for tables given as
    mappings of column name -> array.  Returns the data and the outcome
    weights (None without an outcomes$weights column), in row order."""
    if model_type not in _MODELS:
        raise IngestError(f"unknown model type {model_type!r}")
    model = _MODELS[model_type]
    if model in (D.CLR, D.CPR):
        add_intercept = False
    if model in (D.PR, D.CPR):
        t = _col(outcomes, "time", np.float64)
        if t is None or np.any(t <= 0):
            raise IngestError("time cannot be non-positive")
    outs = sort_outcomes(model, outcomes)
    covs = sort_covariates(model, covariates, outs)
    return load(model, outs, covs, add_intercept), outs["weights"]

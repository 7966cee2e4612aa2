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

Host-side numpy, or (`device=`) the covariate half on the GPU
(cyc_ingest_covariates); the result uploads with `api.Dataset` like any
CyclopsData.
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


def _covariate_columns(covs: dict):
    """loadMultipleX on covariates in the reference's order: (formats,
    row-id offsets, row positions, value offsets, values, covariateIds) of
    the covariate columns, offsets from 0."""
    fmts, ptr, vptr, idx_parts, val_parts, labels = [], [0], [0], [], [], []
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
        nz = None if val is None else val != 0.0
        not01 = None if val is None else ~((val == 0.0) | (val == 1.0))
        for a, b in zip(starts, ends):
            labels.append(int(cid[a]))
            if val is None:
                fmts.append(D.INDICATOR)
                rows, vals = pos[a:b], None
            else:
                keep = nz[a:b]
                sparse = bool(not01[a:b].any())      # first value, or an upcast (:176-184)
                fmts.append(D.SPARSE if sparse else D.INDICATOR)
                rows, vals = pos[a:b][keep], (val[a:b][keep] if sparse else None)
            idx_parts.append(rows.astype(np.int32))
            ptr.append(ptr[-1] + rows.size)
            if vals is not None:
                val_parts.append(vals.astype(np.float64))
            vptr.append(vptr[-1] + (0 if vals is None else vals.size))
    col_idx = np.concatenate(idx_parts) if idx_parts else np.zeros(0, np.int32)
    col_val = np.concatenate(val_parts) if val_parts else np.zeros(0)
    return (np.asarray(fmts, np.int32), np.asarray(ptr, np.int64), col_idx, np.asarray(vptr, np.int64), col_val,
            np.asarray(labels, np.int64))


def _assemble(model: int, outs: dict, cols, add_intercept: bool) -> D.CyclopsData:
    """ModelData::loadY + loadX(intercept) + the Poisson offset in front of
    the covariate columns `cols` (as _covariate_columns returns them)."""
    K = outs["rowId"].size
    # loadY: strata renumbered by runs (:100-122)
    pid = None
    if outs["stratumId"] is not None:
        s = outs["stratumId"]
        pid = np.concatenate([[0], np.cumsum(s[1:] != s[:-1])]).astype(np.int32) if K else np.zeros(0, np.int32)
    fmt, ptr, idx, vptr, val, lab = cols
    offset = model in (D.PR, D.CPR)
    has_intercept = add_intercept and model in (D.LR, D.PR)
    pre_fmt, pre_lab, pre_vptr, pre_val = [], [], [0], []
    if offset:
        t = outs["time"]
        if t is None:
            raise IngestError("Poisson models need outcomes$time")
        # setOffsetCovariate(-1) + logTransformCovariate(0): the C library log, as std::log
        pre_fmt.append(D.DENSE)
        pre_lab.append(-1)
        pre_val.append(np.fromiter(map(math.log, t.tolist()), np.float64, t.size))
        pre_vptr.append(K)
    if has_intercept:
        pre_fmt.append(D.INTERCEPT)                    # loadX(0, none, none): INTERCEPT, to the front
        pre_lab.append(0)
        pre_vptr.append(pre_vptr[-1])
    n_pre = len(pre_fmt)
    col_ptr = np.concatenate([np.zeros(n_pre, np.int64), ptr])
    val_ptr = np.concatenate([np.asarray(pre_vptr, np.int64), vptr[1:] + pre_vptr[-1]])
    col_val = np.concatenate(pre_val + [val]) if pre_val else val
    cd = D.CyclopsData(model=model, y=np.ascontiguousarray(outs["y"]),
                       col_format=np.concatenate([np.asarray(pre_fmt, np.int32), fmt]).astype(np.int32),
                       col_ptr=col_ptr, col_idx=np.ascontiguousarray(idx, np.int32),
                       val_ptr=val_ptr, col_val=np.ascontiguousarray(col_val, np.float64),
                       pid=pid, time=outs["time"], has_offset=offset, has_intercept=has_intercept)
    cd.labels = np.concatenate([np.asarray(pre_lab, np.int64), lab])
    return cd


def load(model: int, outs: dict, covs: dict, add_intercept: bool) -> D.CyclopsData:
    """ModelData::loadY + loadX(intercept) + loadMultipleX + the Poisson
    offset, on tables already in the reference's order."""
    return _assemble(model, outs, _covariate_columns(covs), add_intercept)


def device_covariate_columns(covariates: Mapping, outs: dict, device: int = 0):
    """The covariate columns built on the GPU (cyc_ingest_covariates): the
    same arrays _covariate_columns makes from the host-sorted table, for the
    unsorted covariate table and the sorted outcomes."""
    import ctypes as C
    from . import _native as N
    cid = _col(covariates, "covariateId", np.int64)
    row = _col(covariates, "rowId", np.int64)
    if cid is None or row is None:
        raise IngestError("covariates need covariateId and rowId")
    val = _col(covariates, "covariateValue", np.float64)
    cid, row = np.ascontiguousarray(cid), np.ascontiguousarray(row)
    val = None if val is None else np.ascontiguousarray(val)
    orow = np.ascontiguousarray(outs["rowId"], np.int64)
    L = N.lib()
    h = C.c_void_p()
    rc = L.cyc_ingest_covariates(int(device), int(cid.size), cid.ctypes.data, row.ctypes.data,
                                 None if val is None else val.ctypes.data, int(orow.size), orow.ctypes.data,
                                 C.byref(h))
    if rc != 0:
        msg = L.cyc_last_error().decode()
        if "Repeated" in msg:
            raise IngestError(msg)
        N.check(rc)
    try:
        J, n_idx, n_val = C.c_int(), C.c_longlong(), C.c_longlong()
        N.check(L.cyc_ingest_sizes(h, C.byref(J), C.byref(n_idx), C.byref(n_val)))
        fmt = np.zeros(J.value, np.int32)
        ptr = np.zeros(J.value + 1, np.int64)
        vptr = np.zeros(J.value + 1, np.int64)
        lab = np.zeros(J.value, np.int64)
        idx = np.zeros(n_idx.value, np.int32)
        vals = np.zeros(n_val.value, np.float64)
        N.check(L.cyc_ingest_copy(h, fmt.ctypes.data, ptr.ctypes.data, idx.ctypes.data, vptr.ctypes.data,
                                  vals.ctypes.data, lab.ctypes.data))
    finally:
        L.cyc_ingest_free(h)
    return fmt, ptr, idx, vptr, vals, lab


def convert_to_cyclops_data(outcomes: Mapping, covariates: Mapping, model_type: str = "lr",
                            add_intercept: bool = True,
                            device: Optional[int] = None) -> Tuple[D.CyclopsData, Optional[np.ndarray]]:
    """convertToCyclopsData (R/NewDataConversion.R:94-210) for tables given as
    mappings of column name -> array.  Returns the data and the outcome
    weights (None without an outcomes$weights column), in row order.  With
    `device`, the covariate table is sorted and loaded on that GPU
    (cyc_ingest_covariates; the outcome table, K rows, is sorted here); a
    clr / cpr covariate table that carries its own stratumId column is
    ordered by it, as the reference does, on the host."""
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
    own_strata = model in (D.CLR, D.CPR) and _col(covariates, "stratumId") is not None
    if device is not None and not own_strata:
        cols = device_covariate_columns(covariates, outs, device)
    else:
        cols = _covariate_columns(sort_covariates(model, covariates, outs))
    return _assemble(model, outs, cols, add_intercept), outs["weights"]

"""Ingest of long-format outcome / covariate tables (cyclops_b200/ingest.py)
against the reference's own loader: the committed fixtures were made by the
reference's ModelData::loadY / loadX / loadMultipleX (tests/golden/
make_golden.py, save_ingest), and where the reference library is built here
the same comparison runs on fresh tables.  Row order, column order, column
formats, row ids, values, strata, y, times and the offset / intercept flags
must match bit for bit.  No GPU."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN
from cyclops_b200 import data as D
from cyclops_b200 import ingest

FIELDS = ["col_format", "col_ptr", "col_idx", "val_ptr", "col_val"]


def _check(d, ref):
    for k in FIELDS:
        np.testing.assert_array_equal(getattr(d, k), ref[k], err_msg=k)
    np.testing.assert_array_equal(d.labels, ref["col_label"])
    np.testing.assert_array_equal(d.y, ref["y"])
    if d.pid is None:
        np.testing.assert_array_equal(ref["pid"], np.arange(d.K))
    else:
        np.testing.assert_array_equal(d.pid, ref["pid"])
    if ref.get("time") is not None:
        np.testing.assert_array_equal(d.time, ref["time"])
    assert int(d.has_offset) == int(ref["has_offset"])
    assert int(d.has_intercept) == int(ref["has_intercept"])


def _fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "ingest_*.npz")))


@pytest.mark.parametrize("path", _fixtures(), ids=lambda p: os.path.basename(p)[:-4])
def test_ingest_matches_reference_loader_fixture(path):
    z = np.load(path)
    outcomes = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    cov = {k[4:]: z[k] for k in z.files if k.startswith("cov_")}
    d, _ = ingest.convert_to_cyclops_data(outcomes, cov, str(z["model_type"]))
    ref = {k[4:]: z[k] for k in z.files if k.startswith("ref_")}
    ref.setdefault("time", None)
    _check(d, ref)
    d.validate()


@pytest.mark.parametrize("mt", ["lr", "pr", "clr", "cpr", "cox"])
def test_ingest_matches_live_reference_loader(mt):
    from oracle import oracle as O
    if not O.have_ref():
        pytest.skip("reference library not built here")
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    model = ingest._MODELS[mt]
    for seed in (11, 12):
        outcomes, cov = make_golden.ingest_tables(mt, seed, with_values=(seed % 2 == 1), n=200, m=1500)
        d, _ = ingest.convert_to_cyclops_data(outcomes, cov, mt)
        outs = ingest.sort_outcomes(model, outcomes)
        covs = ingest.sort_covariates(model, cov, outs)
        ref = O.ref_ingest(model, {k: outs[k] for k in ("rowId", "y", "stratumId", "time") if outs[k] is not None},
                           {"rowId": covs["rowId"], "covariateId": covs["covariateId"],
                            "covariateValue": covs["covariateValue"]},
                           mt in ("lr", "pr"), mt in ("pr", "cpr"))
        _check(d, ref)


def test_sort_rules():
    out = {"rowId": np.array([5, 3, 4, 1, 2]), "y": np.array([0., 1., 0., 1., 0.]),
           "stratumId": np.array([2, 1, 2, 1, 2]), "time": np.array([1.0, 2.0, 3.0, 2.0, 3.0])}
    np.testing.assert_array_equal(ingest.sort_outcomes(D.LR, out)["rowId"], [1, 2, 3, 4, 5])
    np.testing.assert_array_equal(ingest.sort_outcomes(D.CLR, out)["rowId"], [1, 3, 2, 4, 5])
    # cox: stratum, time descending, y, rowId
    np.testing.assert_array_equal(ingest.sort_outcomes(D.COX, out)["rowId"], [1, 3, 2, 4, 5])


def test_formats_zero_values_and_upcast():
    out = {"rowId": np.arange(6), "y": np.zeros(6)}
    cov = {"rowId": np.array([0, 2, 4, 1, 3, 0, 5]), "covariateId": np.array([7, 7, 7, 8, 8, 9, 9]),
           "covariateValue": np.array([1.0, 0.0, 1.0, 1.0, 3.5, 0.0, 0.0])}
    d, _ = ingest.convert_to_cyclops_data(out, cov, "lr")
    # intercept, then covariate 7 (indicator, the zero dropped), 8 (upcast to sparse), 9 (all zero: empty)
    np.testing.assert_array_equal(d.col_format, [D.INTERCEPT, D.INDICATOR, D.SPARSE, D.INDICATOR])
    np.testing.assert_array_equal(d.column(1)[0], [0, 4])
    rows, vals = d.column(2)
    np.testing.assert_array_equal(rows, [1, 3])
    np.testing.assert_array_equal(vals, [1.0, 3.5])
    assert d.column(3)[0].size == 0
    np.testing.assert_array_equal(d.labels, [0, 7, 8, 9])


def test_rows_without_outcome_are_dropped_and_errors():
    out = {"rowId": np.array([1, 2]), "y": np.array([0., 1.])}
    d, _ = ingest.convert_to_cyclops_data(out, {"rowId": np.array([1, 9, 2]), "covariateId": np.array([4, 4, 4])}, "lr")
    assert d.nnz == 2
    with pytest.raises(ingest.IngestError, match="Repeated"):
        ingest.convert_to_cyclops_data(out, {"rowId": np.array([1, 1]), "covariateId": np.array([4, 4])}, "lr")
    with pytest.raises(ingest.IngestError, match="non-positive"):
        ingest.convert_to_cyclops_data({**out, "time": np.array([1.0, 0.0])},
                                       {"rowId": np.array([1]), "covariateId": np.array([4])}, "pr")
    with pytest.raises(ingest.IngestError):
        ingest.convert_to_cyclops_data(out, {"rowId": np.array([1]), "covariateId": np.array([4])}, "sccs")


def test_weights_follow_the_row_order():
    out = {"rowId": np.array([3, 1, 2]), "y": np.array([0., 1., 0.]), "weights": np.array([0.3, 0.1, 0.2])}
    _, w = ingest.convert_to_cyclops_data(out, {"rowId": np.array([1]), "covariateId": np.array([4])}, "lr")
    np.testing.assert_array_equal(w, [0.1, 0.2, 0.3])

"""Device ingest (cyc_ingest_covariates through ingest.convert_to_cyclops_data
with device=0) against the host ingest, which the reference's own loader
pins (tests/test_ingest.py): every array of the resulting column store --
formats, row-id offsets, row positions, value offsets, values, labels, y,
strata, times, offset and intercept flags -- equal bit for bit, on the
reference-made fixtures and on larger tables with the awkward cases
(unsorted rowIds, covariate rows without an outcome, repeated outcome
rowIds, zero values, indicator columns upcast to sparse, tied Cox times,
empty and all-dropped tables), and the repeated-entry error."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN
from cyclops_b200 import data as D
from cyclops_b200 import ingest

pytestmark = pytest.mark.gpu

FIELDS = ["col_format", "col_ptr", "col_idx", "val_ptr", "col_val", "labels", "y"]


def _same(a, b):
    for k in FIELDS:
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
        assert getattr(a, k).dtype == getattr(b, k).dtype, k
    for k in ("pid", "time"):
        x, y = getattr(a, k), getattr(b, k)
        assert (x is None) == (y is None), k
        if x is not None:
            np.testing.assert_array_equal(x, y, err_msg=k)
    assert a.has_offset == b.has_offset and a.has_intercept == b.has_intercept


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ingest_*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_device_ingest_matches_reference_fixture(cuda_lib, path):
    z = np.load(path)
    outcomes = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    cov = {k[4:]: z[k] for k in z.files if k.startswith("cov_")}
    host, _ = ingest.convert_to_cyclops_data(outcomes, cov, str(z["model_type"]))
    dev, _ = ingest.convert_to_cyclops_data(outcomes, cov, str(z["model_type"]), device=0)
    _same(dev, host)
    np.testing.assert_array_equal(dev.col_format, z["ref_col_format"])
    np.testing.assert_array_equal(dev.col_idx, z["ref_col_idx"])


def _tables(mt, seed, n, m, values=True, dup_outcomes=False):
    rng = np.random.default_rng(seed)
    rid = rng.permutation(np.arange(5_000, 5_000 + n)).astype(np.int64)
    if dup_outcomes:                                    # a few rowIds twice: the last one wins
        rid[rng.choice(n, n // 50, replace=False)] = rid[rng.choice(n, n // 50, replace=False)]
    outcomes = {"rowId": rid, "y": rng.integers(0, 2, n).astype(np.float64),
                "stratumId": rng.integers(0, max(2, n // 5), n).astype(np.int64),
                "time": rng.choice([0.25, 0.5, 1.0, 2.0, 3.0, 7.5], n).astype(np.float64)}
    rows = rng.integers(4_900, 5_000 + n, m).astype(np.int64)          # some without an outcome
    cids = (rng.zipf(1.3, m) % 400 + rng.integers(0, 3, m) * 1_000_003).astype(np.int64)
    _, u = np.unique(rows * 10_000_000_000 + cids, return_index=True)
    u = rng.permutation(u)
    cov = {"rowId": rows[u], "covariateId": cids[u]}
    if values:
        cov["covariateValue"] = rng.choice([0.0, 1.0, 1.0, 1.0, 1.0, 2.5, -0.75], u.size).astype(np.float64)
    return outcomes, cov


@pytest.mark.parametrize("mt", ["lr", "pr", "clr", "cpr", "cox"])
@pytest.mark.parametrize("values", [True, False])
def test_device_ingest_matches_host(cuda_lib, mt, values):
    for seed, (n, m) in enumerate([(300, 3_000), (20_000, 400_000)]):
        outcomes, cov = _tables(mt, 100 + seed, n, m, values=values, dup_outcomes=(seed == 1))
        host, wh = ingest.convert_to_cyclops_data(outcomes, cov, mt)
        dev, wd = ingest.convert_to_cyclops_data(outcomes, cov, mt, device=0)
        _same(dev, host)
        dev.validate()


def test_device_ingest_edges(cuda_lib):
    out = {"rowId": np.arange(6), "y": np.zeros(6)}
    cov = {"rowId": np.array([0, 2, 4, 1, 3, 0, 5]), "covariateId": np.array([7, 7, 7, 8, 8, 9, 9]),
           "covariateValue": np.array([1.0, 0.0, 1.0, 1.0, 3.5, 0.0, 0.0])}
    dev, _ = ingest.convert_to_cyclops_data(out, cov, "lr", device=0)
    host, _ = ingest.convert_to_cyclops_data(out, cov, "lr")
    _same(dev, host)
    np.testing.assert_array_equal(dev.col_format, [D.INTERCEPT, D.INDICATOR, D.SPARSE, D.INDICATOR])
    # no covariate rows, and none with an outcome
    for c in ({"rowId": np.zeros(0, np.int64), "covariateId": np.zeros(0, np.int64)},
              {"rowId": np.array([99, 98]), "covariateId": np.array([4, 5])}):
        _same(ingest.convert_to_cyclops_data(out, c, "lr", device=0)[0], ingest.convert_to_cyclops_data(out, c, "lr")[0])
    with pytest.raises(ingest.IngestError, match="Repeated row-column entry at 1 - 4"):
        ingest.convert_to_cyclops_data({"rowId": np.array([1, 2]), "y": np.array([0., 1.])},
                                       {"rowId": np.array([2, 1, 1]), "covariateId": np.array([4, 4, 4])}, "lr",
                                       device=0)


def test_device_ingest_fits_like_host_ingest(cuda_lib):
    """The fit of device-ingested data is the fit of host-ingested data."""
    from cyclops_b200 import api
    outcomes, cov = _tables("lr", 7, 5_000, 60_000)
    host, _ = ingest.convert_to_cyclops_data(outcomes, cov, "lr")
    dev, _ = ingest.convert_to_cyclops_data(outcomes, cov, "lr", device=0)
    prior = api.PriorSpec(D.PRIOR_LAPLACE, 1.0, [0])
    a = api.fit_cyclops_model(dev, prior, api.create_control())
    b = api.fit_cyclops_model(host, prior, api.create_control())
    assert np.array_equal(a.beta, b.beta) and a.iterations == b.iterations

"""Host-side data rules: ingest order, sort orders, strata renumbering, fold
intervals.  No GPU."""
import numpy as np
import pytest

from conftest import GOLDEN
from cyclops_b200 import data as D


def test_cox_rows_sorted_by_stratum_desc_time_then_y():
    d = D.synth_cox(K=4000, P=20, density=0.05, n_strata=7, seed=5, ties=1)
    key = list(zip(d.pid, -d.time, d.y))
    assert key == sorted(key)                      # order(pid, -time, y)
    d.validate()


def test_conditional_rows_grouped_by_stratum():
    d = D.synth_conditional(K=1000, P=30, density=0.05, seed=6)
    assert np.all(np.diff(d.pid) >= 0)
    s = d.strata()
    assert s[0] == 0 and s[-1] == 199
    assert np.all(np.bincount(s) == 5)


def test_strata_renumbered_by_runs():
    d = D.ColumnBuilder(6).intercept().build(D.CLR, np.zeros(6), pid=np.array([7, 7, 3, 3, 7, 9]))
    np.testing.assert_array_equal(d.strata(), [0, 0, 1, 1, 2, 3])


def test_column_order_offset_then_dense_then_indicator():
    d = D.synth_poisson(K=2000, P=50, per_row=4, n_dense=3, seed=7)
    assert list(d.col_format[:5]) == [D.DENSE] * 5        # offset, intercept, 3 dense
    assert set(d.col_format[5:]) == {D.INDICATOR}
    np.testing.assert_allclose(d.column(0)[1], d.time)
    np.testing.assert_allclose(d.column(1)[1], 1.0)
    d.validate()


def test_zipf_rows_distinct_and_per_row_count():
    indptr, rows = D._zipf_rows_without_replacement(np.random.default_rng(0), 500, 300, 10, 1.1)
    cols = np.repeat(np.arange(300), np.diff(indptr))
    pairs = set(zip(rows.tolist(), cols.tolist()))
    assert len(pairs) == rows.shape[0]                     # no duplicate (row, col)
    assert np.all(np.bincount(rows, minlength=500) == 10)


def test_validate_rejects_unsorted_rows():
    b = D.ColumnBuilder(5)
    b.fmt.append(D.INDICATOR)
    b.idx.append(np.array([3, 1], np.int32))
    b.val.append(np.zeros(0))
    d = b.build(D.LR, np.zeros(5))
    with pytest.raises(ValueError):
        d.validate()


def test_fold_interval_sizes_match_reference_rule():
    z = np.load(GOLDEN + "/cv_folds.npz")
    K = int(z["K"])
    held = (z["by_row"] == 0).sum(axis=1)
    ours = (D.cv_fold_weights(K, 10, 1) == 0).sum(axis=1)
    np.testing.assert_array_equal(held[:10], ours)
    # each repetition partitions the rows
    np.testing.assert_array_equal((z["by_row"][:10] == 0).sum(axis=0), np.ones(K))


def test_lambda_grid_and_variance():
    g = D.lambda_grid(1e-4, 1.0, 20)
    assert g[0] == pytest.approx(1e-4) and g[-1] == pytest.approx(1.0)
    assert np.allclose(np.diff(np.log(g)), np.log(1e4) / 19)
    assert D.laplace_variance(0.1) == pytest.approx(200.0)


def test_library_fold_masks_equal_reference_selector(cuda_lib):
    """cyc_cv_fold_weights is host code: bit-exact against the masks the
    reference's CrossValidationSelector produced (no GPU involved)."""
    from cyclops_b200 import api
    z = np.load(GOLDEN + "/cv_folds.npz")
    K = int(z["K"])
    np.testing.assert_array_equal(api.cv_fold_weights(K, 10, int(z["seed_row"]), n_reps=2), z["by_row"])
    np.testing.assert_array_equal(api.cv_fold_weights(K, 5, int(z["seed_pid"]), ids=z["pid"]), z["by_pid"])


def test_library_bootstrap_weights_equal_reference_selector(cuda_lib):
    """cyc_bootstrap_weights is host code: bit-exact against the replicate
    weights the reference's BootstrapSelector drew (one permute in its
    constructor, one per replicate), per row and by matched stratum."""
    from cyclops_b200 import api
    z = np.load(GOLDEN + "/bootstrap_weights.npz")
    K = int(z["K"])
    np.testing.assert_array_equal(api.bootstrap_weights(K, 8, int(z["seed_row"])), z["by_row"])
    np.testing.assert_array_equal(api.bootstrap_weights(K, 4, int(z["seed_pid"]), ids=z["pid"]), z["by_pid"])
    assert np.all(z["by_row"].sum(axis=1) == K)          # K draws with replacement per replicate

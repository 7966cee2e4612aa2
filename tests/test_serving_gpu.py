"""Serving on the GPU: the same requests served one at a time and as an
overlapping mix (several fits on the device at once, some requests batched
on a shared dataset) give the same results.  A fit is deterministic and
independent of what else runs, so a request that runs alone in both is
identical; a request batched with others in the mix follows the same CCD
and agrees within the precision contract (beta 1e-6 relative)."""
import numpy as np
import pytest

from conftest import assert_contract
from cyclops_b200 import api, serving
from cyclops_b200 import data as D

pytestmark = pytest.mark.gpu


def _requests():
    reqs = []
    rng = np.random.default_rng(11)
    for i in range(8):
        model = [D.LR, D.PR, D.CLR][i % 3]
        K = int(rng.integers(2_000, 20_000))
        K -= K % 5
        P = int(rng.integers(100, 600))
        data = serving.synth_request_data(model, K, P, 0.01, seed=100 + i)
        lam = float(np.exp(rng.uniform(np.log(1e-2), np.log(1.0))))
        reqs.append(serving.Request(i, data, api.PriorSpec(D.PRIOR_LAPLACE, D.laplace_variance(lam)),
                                    api.create_control(), 0.0))
    shared = serving.synth_request_data(D.LR, 15_000, 300, 0.01, seed=999)
    for j, lam in enumerate([0.05, 0.1, 0.3, 0.6]):
        reqs.append(serving.Request(8 + j, shared, api.PriorSpec(D.PRIOR_LAPLACE, D.laplace_variance(lam)),
                                    api.create_control(), 0.0, key="shared"))
    return reqs


def test_alone_and_in_the_mix_agree(cuda_lib):
    reqs = _requests()
    alone = serving.Server(slots=1, max_batch=1).run(reqs, realtime=False)
    mix = serving.Server(slots=4, max_batch=8).run(reqs, realtime=False)
    assert all(r.error is None for r in alone + mix), [r.error for r in alone + mix if r.error]
    assert max(r.batch_size for r in mix) == 4          # the shared-dataset requests ran as one batch
    for a, m in zip(alone, mix):
        assert a.rid == m.rid and a.return_flag == m.return_flag == 0
        if m.batch_size == 1:
            assert np.array_equal(a.beta, m.beta), a.rid
            assert a.iterations == m.iterations
        else:
            err = np.max(np.abs(a.beta - m.beta) / np.maximum(np.abs(a.beta), 1.0))
            assert err < 1e-6, (a.rid, err)
            np.testing.assert_array_equal(a.beta != 0, m.beta != 0)
            assert a.iterations == m.iterations


def test_served_fit_is_the_library_fit(cuda_lib):
    """A request served alone runs the persistent kernel on one fit; it is the
    device fit of cyc_fit to the precision contract, with the same cycles."""
    reqs = _requests()[:3]
    res = serving.Server(slots=3).run(reqs, realtime=False)
    for r, q in zip(res, reqs):
        ref = api.fit_cyclops_model(q.data, q.prior, q.control)
        err = np.max(np.abs(r.beta - ref.beta) / np.maximum(np.abs(ref.beta), 1.0))
        assert err < 1e-6, err
        assert r.iterations == ref.iterations


def test_served_fits_match_oracle(cuda_lib):
    """Every request of the mix (overlapping on the device, the shared-data
    requests batched together) against the restatement oracle fitting the
    same data, prior and control on its own: the precision contract."""
    from oracle import oracle as O
    reqs = _requests()
    mix = serving.Server(slots=4, max_batch=8).run(reqs, realtime=False)
    for r, q in zip(mix, reqs):
        assert r.error is None, r.error
        ctl = O.make_control(tolerance=q.control.tolerance, max_iterations=q.control.max_iterations,
                             convergence_type=q.control.convergence_type)
        ref = O.port().fit(q.data, q.prior.prior_type, q.prior.variance, control=ctl,
                           exclude=api._exclude_for(q.data, q.prior), weights=q.weights)
        assert_contract(r, ref, what=r.rid)

"""Serving scheduler (cyclops_b200/serving.py), host logic only: the fits are
replaced by a stand-in that records what was admitted and when.  No GPU."""
import threading
import time

import numpy as np

from cyclops_b200 import api, serving
from cyclops_b200 import data as D


def _req(rid, arrival=0.0, key=None, K=1000, P=50, variance=1.0, data=None):
    d = data or D.synth_logistic(K=K, P=P, density=0.02, n_true=5, seed=rid + 1)
    return serving.Request(rid, d, api.PriorSpec(D.PRIOR_LAPLACE, variance), api.create_control(), arrival, key=key)


class Recorder(serving.Server):
    """Runs no fit: each job sleeps `hold` seconds and records the jobs that
    were running at the same time."""

    def __init__(self, hold=0.05, **kw):
        super().__init__(**kw)
        self.hold = hold
        self.lock = threading.Lock()
        self.running = 0
        self.max_running = 0
        self.jobs = []

    def _run_job(self, job, admitted, t0):
        with self.lock:
            self.running += 1
            self.max_running = max(self.max_running, self.running)
            self.jobs.append([r.rid for r in job])
        time.sleep(self.hold)
        with self.lock:
            self.running -= 1
        now = time.monotonic() - t0
        return [serving.Response(r.rid, np.zeros(r.data.J), 0.0, 1, 0, r.arrival, admitted, now, len(job))
                for r in job]


def test_admits_in_arrival_order_within_the_slot_limit():
    reqs = [_req(i, arrival=0.0) for i in range(10)]
    srv = Recorder(slots=3, max_batch=1)
    res = srv.run(reqs, realtime=False)
    assert [r.rid for r in res] == list(range(10))
    assert srv.max_running == 3
    assert [j[0] for j in srv.jobs] == list(range(10))           # first come, first admitted
    assert all(r.error is None and r.finished >= r.admitted >= r.arrival for r in res)


def test_budget_holds_back_requests_until_memory_frees():
    reqs = [_req(i) for i in range(6)]
    one = serving.request_bytes(reqs[0].data)
    srv = Recorder(slots=6, max_batch=1, budget_bytes=2 * one + 1)
    srv.run(reqs, realtime=False)
    assert srv.max_running == 2


def test_request_over_budget_is_rejected_not_stalled():
    big = _req(0, K=20000, P=200)
    small = _req(1)
    srv = Recorder(slots=2, max_batch=1, budget_bytes=serving.request_bytes(small.data) + 1)
    res = srv.run([big, small], realtime=False)
    assert res[0].error and "budget" in res[0].error
    assert res[1].error is None


def test_requests_sharing_a_dataset_batch_together():
    shared = D.synth_logistic(K=1000, P=40, density=0.05, n_true=5, seed=3)
    reqs = [_req(i, key="grid", data=shared, variance=1.0 + i) for i in range(5)] + [_req(5)]
    srv = Recorder(slots=1, max_batch=4)
    res = srv.run(reqs, realtime=False)
    assert srv.jobs[0] == [0, 1, 2, 3] and srv.jobs[1] == [4] and srv.jobs[2] == [5]
    assert [r.batch_size for r in res] == [4, 4, 4, 4, 1, 1]


def test_realtime_arrivals_wait_for_their_time():
    reqs = [_req(i, arrival=0.05 * i) for i in range(4)]
    srv = Recorder(slots=4, hold=0.01)
    res = srv.run(reqs, realtime=True)
    for r in res:
        assert r.admitted >= r.arrival - 1e-3
        assert r.latency >= 0.0


def test_request_stream_shapes():
    reqs = serving.request_stream(30, rate=50.0, seed=3, max_entries=200_000)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0)
    models = {r.data.model for r in reqs}
    assert models <= {D.LR, D.PR, D.CLR}
    for r in reqs:
        assert 1000 - 5 <= r.data.K <= 2_000_000
        assert r.data.col_idx.size <= 200_000 * 1.2 + 100
        lam = np.sqrt(2.0 / r.prior.variance)
        assert 1e-3 <= lam <= 1.0
    s = serving.summarize([serving.Response(0, None, 0.0, 1, 0, 0.0, 0.1, 0.3, 1)], 1.0)
    assert abs(s["latency_p50_s"] - 0.3) < 1e-12


def test_deadline_answers_the_rest():
    reqs = [_req(i, arrival=0.0) for i in range(6)]
    srv = Recorder(slots=1, hold=0.1)
    res = srv.run(reqs, realtime=True, deadline=0.15)
    served = [r for r in res if r.error is None]
    late = [r for r in res if r.error == "not admitted before the deadline"]
    assert len(served) >= 1 and len(late) >= 1 and len(served) + len(late) == 6
    assert serving.summarize(res, 1.0)["not_admitted"] == len(late)

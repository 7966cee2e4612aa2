"""Serving: a stream of fit requests on one GPU, continuously admitted.

Each request is one fit (data, prior, control) with an arrival time.  The
scheduler admits queued requests in arrival order as soon as a fit slot and
the device-memory budget allow, so requests that arrive while others run
start without waiting for them; each slot is a worker thread whose fit runs
on its own CUDA stream, so admitted fits overlap on the device.  A fit runs
as one persistent launch of the batched solver (`cyc_batch_fit`, one fit or
several), or, for what that solver does not cover (Cox, Zhang-Oles
convergence), as `cyc_fit`.  Requests that share one dataset and prior type (a
`key`) are admitted together as one batched solve (`cyc_batch_fit`), up to
`max_batch` at a time.  Memory is returned when a fit finishes.

Latency is wall-clock from a request's arrival to its result; the run
reports p50 / p99 and fits per second.  A result does not depend on what
else runs: single fits are deterministic and independent of one another, and
a batched fit follows the same CCD as the single one (the test compares
both).

    python -m cyclops_b200.serving [--requests 200 --rate 50 --slots 16 --max-seconds 300]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from typing import Any, List, Optional, Sequence

import numpy as np

from . import api
from . import data as D


@dataclasses.dataclass
class Request:
    rid: int
    data: D.CyclopsData
    prior: api.PriorSpec
    control: api.ControlSpec
    arrival: float = 0.0                 # seconds after the stream starts
    weights: Optional[np.ndarray] = None
    key: Any = None                      # requests with one key share `data` and may batch


@dataclasses.dataclass
class Response:
    rid: int
    beta: Optional[np.ndarray]
    log_likelihood: float
    iterations: int
    return_flag: int
    arrival: float
    admitted: float
    finished: float
    batch_size: int
    error: Optional[str] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def request_bytes(data: D.CyclopsData, fits: int = 1) -> int:
    """Device bytes a request holds while it runs: the dataset (row ids,
    values, the row-major copy, per-row arrays) and the per-fit solver state
    (linear predictor, its saved copy, exp, weights, denominators; beta,
    trust region and XjY per column)."""
    K, J = data.K, data.J
    nnz_idx = int(data.col_idx.size)
    nnz_val = int(data.col_val.size)
    dataset = nnz_idx * 4 + nnz_val * 8 + J * 24 + K * 24 + (nnz_idx + nnz_val) * 12 + K * 8
    state = fits * (K * 8 * 6 + J * 8 * 4)
    return int(1.25 * (dataset + state)) + (1 << 20)


def _persistent_ok(r: Request) -> bool:
    """Requests the persistent batched kernel serves (also when alone: one
    launch for the whole fit instead of kernels per coordinate, measured
    2.5-14x faster on B200 with the same iterations and beta to ~1e-15):
    lr, pr, clr, cpr under gradient, mittal or lange convergence."""
    return r.data.model in (D.LR, D.PR, D.CLR, D.CPR) and \
        r.control.convergence_type in (D.CONV_GRADIENT, D.CONV_MITTAL, D.CONV_LANGE)


class Server:
    def __init__(self, device: int = 0, slots: int = 16, budget_bytes: Optional[int] = None, max_batch: int = 8):
        self.device = device
        self.slots = slots
        self.max_batch = max_batch
        if budget_bytes is None:
            budget_bytes = 64 << 30
        self.budget = budget_bytes

    # one admitted job: a single fit, or a batch of requests on one dataset
    def _run_job(self, job: List[Request], admitted: float, t0: float) -> List[Response]:
        out = []
        try:
            ds = api.Dataset(job[0].data, self.device)
            try:
                if len(job) == 1 and not _persistent_ok(job[0]):
                    r = job[0]
                    fits = [api.fit_cyclops_model(ds, r.prior, r.control, weights=r.weights)]
                else:
                    prior = job[0].prior
                    fits = api.batch_fit(ds, prior, [r.prior.variance for r in job],
                                         [r.weights for r in job], job[0].control)
            finally:
                ds.close()
            now = time.monotonic() - t0
            for r, f in zip(job, fits):
                out.append(Response(r.rid, f.beta, f.log_likelihood, f.iterations, f.return_flag, r.arrival,
                                    admitted, now, len(job)))
        except Exception as e:          # reported per request, the server goes on
            now = time.monotonic() - t0
            for r in job:
                out.append(Response(r.rid, None, math.nan, 0, -1, r.arrival, admitted, now, len(job), str(e)))
        return out

    def run(self, requests: Sequence[Request], realtime: bool = True,
            deadline: Optional[float] = None) -> List[Response]:
        """Serve `requests` (arrival times in seconds from now when `realtime`,
        otherwise all present at once) and return one response per request.
        Requests not admitted `deadline` seconds after the start are answered
        with an error instead (the fits already running finish)."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        queue: List[Request] = []
        results: List[Response] = []
        cond = threading.Condition()
        state = {"free": self.slots, "bytes": 0}
        t0 = time.monotonic()

        def done(fut, nbytes):
            res = fut.result()
            with cond:
                results.extend(res)
                state["free"] += 1
                state["bytes"] -= nbytes
                cond.notify_all()

        with ThreadPoolExecutor(max_workers=self.slots) as pool:
            i = 0
            while True:
                with cond:
                    now = time.monotonic() - t0
                    while i < len(pending) and (not realtime or pending[i].arrival <= now):
                        queue.append(pending[i])
                        i += 1
                    if deadline is not None and now > deadline:
                        for r in queue + list(pending[i:]):
                            results.append(Response(r.rid, None, math.nan, 0, -1, r.arrival, now, now, 1,
                                                    "not admitted before the deadline"))
                        queue.clear()
                        i = len(pending)
                    # admit in arrival order while a slot and the budget allow
                    while queue and state["free"] > 0:
                        head = queue[0]
                        job = [head]
                        if head.key is not None:
                            for r in queue[1:]:
                                if len(job) >= self.max_batch:
                                    break
                                if r.key == head.key and r.prior.prior_type == head.prior.prior_type \
                                        and r.control == head.control:
                                    job.append(r)
                        nbytes = request_bytes(head.data, len(job))
                        if nbytes > self.budget:
                            for r in job:
                                results.append(Response(r.rid, None, math.nan, 0, -1, r.arrival, now, now, len(job),
                                                        "request larger than the device-memory budget"))
                                queue.remove(r)
                            continue
                        if state["bytes"] + nbytes > self.budget:
                            break
                        for r in job:
                            queue.remove(r)
                        state["free"] -= 1
                        state["bytes"] += nbytes
                        fut = pool.submit(self._run_job, job, now, t0)
                        fut.add_done_callback(lambda f, nb=nbytes: done(f, nb))
                    if i >= len(pending) and not queue and state["free"] == self.slots:
                        break
                    wait = None
                    if i < len(pending) and realtime:
                        wait = max(0.0, pending[i].arrival - (time.monotonic() - t0))
                    cond.wait(timeout=wait if wait is not None else 1.0)
        results.sort(key=lambda r: r.rid)
        return results


# --------------------------------------------------------------------------
# the request stream of the serving benchmark
# --------------------------------------------------------------------------

def synth_request_data(model: int, K: int, P: int, density: float, seed: int) -> D.CyclopsData:
    """One request's data: an intercept (lr, pr) and P indicator columns at
    the given density (uniform), y from a sparse true beta; clr uses 1:4
    matched strata (stratum of 5 rows, one case)."""
    if model == D.CLR:
        return D.synth_conditional(K=K, P=P, density=density, stratum_size=5, n_true=min(30, P), seed=seed)
    if model == D.LR:
        return D.synth_logistic(K=K, P=P, density=density, n_true=min(50, P), intercept=-1.0, seed=seed)
    rng = np.random.default_rng(seed)
    indptr, indices = D._bernoulli_csc(rng, K, P, density)
    beta = np.zeros(P)
    cols = rng.choice(P, size=min(50, P), replace=False)
    beta[cols] = rng.normal(0.0, 0.3, size=cols.shape[0])
    eta = -1.0 + D._csc_matvec(indptr, indices, beta, K)
    y = rng.poisson(np.exp(np.minimum(eta, 5.0))).astype(np.float64)
    return D.ColumnBuilder(K).intercept().indicator_csc(indptr, indices).build(D.PR, y, has_intercept=True)


def request_stream(n: int, rate: float, seed: int = 7, max_entries: int = 4_000_000) -> List[Request]:
    """The serving stream: Poisson arrivals at `rate`/s; rows log-uniform in
    1k..2M, columns log-uniform in 100..100k, indicator density U(0.1 %,
    2 %); 60 % logistic, 25 % Poisson, 15 % conditional logistic (1:4
    matched); Laplace lambda log-uniform in 1e-3..1.  Requests whose stored
    entries would exceed `max_entries` have their density scaled down to that
    many (host-side generation time and memory; the sizes stay as drawn)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        K = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e6)))))
        P = int(round(math.exp(rng.uniform(math.log(100), math.log(1e5)))))
        density = rng.uniform(0.001, 0.02)
        u = rng.random()
        model = D.LR if u < 0.6 else (D.PR if u < 0.85 else D.CLR)
        if model == D.CLR:
            K = max(10, K - K % 5)
        if K * P * density > max_entries:
            density = max_entries / (K * P)
        lam = math.exp(rng.uniform(math.log(1e-3), math.log(1.0)))
        data = synth_request_data(model, K, P, density, seed=int(rng.integers(1 << 30)))
        prior = api.PriorSpec(D.PRIOR_LAPLACE, D.laplace_variance(lam))
        out.append(Request(i, data, prior, api.create_control(), arrival=t))
    return out


def summarize(res: Sequence[Response], wall: float) -> dict:
    ok = [r for r in res if r.error is None]
    lat = np.array([r.latency for r in ok]) if ok else np.zeros(1)
    return {
        "requests": len(res), "completed": len(ok), "errors": len(res) - len(ok),
        "not_admitted": int(sum(r.error == "not admitted before the deadline" for r in res)),
        "converged": int(sum(r.return_flag == 0 for r in ok)),
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "latency_mean_s": float(lat.mean()), "wall_s": wall, "fits_per_s": len(ok) / wall if wall > 0 else None,
        "batched_requests": int(sum(r.batch_size > 1 for r in ok)),
        # time on the device once admitted, and how many fits ran at once on average
        "service_p50_s": float(np.percentile([r.finished - r.admitted for r in ok], 50)) if ok else None,
        "service_p99_s": float(np.percentile([r.finished - r.admitted for r in ok], 99)) if ok else None,
        "mean_concurrency": float(sum(r.finished - r.admitted for r in ok) / wall) if ok and wall > 0 else None,
        "cycles_p50": float(np.percentile([r.iterations for r in ok], 50)) if ok else None,
        "cycles_max": int(max(r.iterations for r in ok)) if ok else None,
    }


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--requests", type=int, default=200)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--slots", type=int, default=16)
    ap.add_argument("--budget-gb", type=float, default=64.0)
    ap.add_argument("--max-entries", type=int, default=4_000_000)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--max-seconds", type=float, default=None,
                    help="stop admitting after this many seconds (the report counts the rest as not served)")
    args = ap.parse_args(argv)
    t = time.time()
    reqs = request_stream(args.requests, args.rate, args.seed, args.max_entries)
    gen = time.time() - t
    server = Server(slots=args.slots, budget_bytes=int(args.budget_gb * (1 << 30)))
    t = time.monotonic()
    res = server.run(reqs, realtime=True, deadline=args.max_seconds)
    wall = time.monotonic() - t
    out = summarize(res, wall)
    out.update({"stream": {"requests": args.requests, "rate_per_s": args.rate, "seed": args.seed,
                           "max_entries": args.max_entries, "generation_s": gen},
                "slots": args.slots, "budget_gb": args.budget_gb,
                "entries_total": int(sum(int(r.data.col_idx.size) for r in reqs))})
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())

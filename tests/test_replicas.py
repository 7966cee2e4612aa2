"""The N > 1 path of bench.py as two gloo ranks on CPU: independent replicas,
one fold seed per rank (different CV folds, each drawn by the reference
selector's rule), the barriers and the max over ranks of the timed region,
and the whole-job rate computed from the slowest rank.  No GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    rep = bench.Replicas("gloo", timeout_s=60)
    folds = bench.fold_ids(1000, rep.fold_seed(bench.FOLD_SEED))
    rep.barrier()
    ms = rep.max(100.0 + 50.0 * rank)            # this rank's "device time"
    rate = rep.total_rate(200, 2, ms)
    rep.close()
    out.put((rank, folds.tolist(), ms, rate))


def test_two_gloo_replicas():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, folds, ms, rate = q.get(timeout=120)
        res[r] = (np.array(folds), ms, rate)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # each rank has its own folds, each a partition of the rows into 10 folds
    assert not np.array_equal(res[0][0], res[1][0])
    for r in range(world):
        assert sorted(set(res[r][0].tolist())) == list(range(10))
    # the timed region is the slowest rank's, the same on every rank
    assert res[0][1] == res[1][1] == 150.0
    assert res[0][2] == pytest.approx(200 * 2 * 2 / 0.150)


def test_single_process_needs_no_group():
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    rep = bench.Replicas("gloo")
    assert rep.world == 1 and rep.dist is None
    assert rep.max(3.0) == 3.0
    assert rep.total_rate(200, 2, 1000.0) == 400.0
    rep.close()

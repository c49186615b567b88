"""The N>1 path of the bench (replicas only) on CPU: two gloo ranks deal a
request list, each rank's share is disjoint and complete together, and the
reductions give the slowest rank's time and the job's total."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws),
                      RANK=str(rank), LOCAL_RANK=str(rank))
    from ndyn_omp_b200 import replicas as R
    w, r, _ = R.init(timeout_s=30)
    assert (w, r) == (ws, rank)
    mine = R.shard(range(11), r, w)
    t = R.reduce_max(1.5 + r, w)          # rank times 1.5 and 2.5 s
    n = R.reduce_sum(len(mine), w)
    R.barrier(w)
    out.put((r, mine, t, n))
    R.finish(w)


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, a, t0, n0), (r1, b, t1, n1) = res
    assert sorted(a + b) == list(range(11)) and not set(a) & set(b)
    assert t0 == t1 == pytest.approx(2.5)
    assert n0 == n1 == 11


def test_single_rank_needs_no_process_group():
    from ndyn_omp_b200 import replicas as R
    assert R.reduce_max(3.0, 1) == 3.0
    assert R.shard([1, 2, 3], 0, 1) == [1, 2, 3]

"""Serving loop (continuous batching): admission by HBM budget, runs that
join while others are on the GPU, and results that do not depend on the mix.

Bars: in mixed precision a run's final state and write_thermo rows are the
same bits whether it ran alone through ndg_run, alone in a server, or in a
server together with other runs that arrived before, with and after it
(the fixed-point force sums and per-system reductions do not depend on the
batch); the admission rule is checked on the host alone.
"""
import numpy as np
import pytest

nd = pytest.importorskip("ndyn_omp_b200")
from ndyn_omp_b200 import workloads as W  # noqa: E402


def test_admit_plan_order_and_budget():
    # in queue order; a request that does not fit keeps waiting, later
    # smaller ones may pass it; the resident bytes count against the budget
    adm = nd.admit_plan([40, 70, 20, 10, 5], budget=100, in_use=10)
    assert adm.tolist() == [True, False, True, True, True]
    assert nd.admit_plan([101], budget=100).tolist() == [False]
    assert nd.admit_plan([], budget=100).tolist() == []
    assert nd.admit_plan([50, 50], budget=100, in_use=100).tolist() == [False, False]


def _requests():
    cu = W.cu_crystal(5, 900.0, seed=41, quirk="fixed")                   # 500 atoms, NVE
    ar = W.ar_liquid(6, 150.0, seed=42, quirk="fixed")                    # 864 atoms, NVT
    na = W.nacl_solid((4, 4, 4), 600.0, seed=43, quirk="fixed")           # 512 atoms, NPT
    cu2 = W.cu_crystal(7, 1400.0, seed=44, quirk="fixed")                 # 1372 atoms, NVE
    for s in (cu, ar, na, cu2):
        s["control"] = dict(s["control"], out_steps=20)
    return [(cu, 130), (ar, 170), (na, 90), (cu2, 210)]


def _estimate(spec):
    """the server's device-bytes estimate of a request (ndg_system_bytes at
    the system's density and rcut + skin)"""
    n = len(spec["typ"])
    rc = max(p[4][0] for p in spec["pairs"])
    skin = spec["control"]["skin"]
    skin = 0.2 * rc if skin < 0 else skin
    return nd.lib().ndg_system_bytes(n, len(spec["masses"]), len(spec["pairs"]), 1000,
                                     n / float(np.prod(spec["box"])), rc + skin, 1)


def _alone_run(spec, nsteps):
    with nd.Context(0, "mixed") as ctx:
        sid = W.add_to_context(ctx, spec)
        rows = ctx.run(nsteps)
        return ctx.state(sid), rows


def _same(a, b):
    (pa, va, aa, ba), ra = a
    (pb, vb, ab, bb), rb = b
    for x, y in ((pa, pb), (va, vb), (aa, ab), (ba, bb)):
        assert np.array_equal(x, y)
    key = ("step", "pe", "ke", "eerr", "press", "vol")
    assert [tuple(r[k] for k in key) for r in ra] == [tuple(r[k] for k in key) for r in rb]


@pytest.mark.gpu
def test_serving_result_same_alone_and_in_mix():
    reqs = _requests()
    alone = [_alone_run(s, n) for s, n in reqs]
    with nd.Server(0, "mixed", hbm_budget=8e9, block_steps=40) as srv:
        t = [W.submit_to_server(srv, reqs[0][0], reqs[0][1]),
             W.submit_to_server(srv, reqs[1][0], reqs[1][1])]
        srv.step()                      # runs 0 and 1 on the GPU
        t.append(W.submit_to_server(srv, reqs[2][0], reqs[2][1]))
        srv.step()                      # run 2 joins the running batch
        srv.step()
        t.append(W.submit_to_server(srv, reqs[3][0], reqs[3][1]))
        done = set()
        for _ in range(40):
            srv.step()
            done |= set(srv.poll())
            if len(done | set(x for x in t if srv.status(x) == 2)) == len(t):
                break
        assert all(srv.status(x) == 2 for x in t)
        st = srv.stats()
        assert st["completed"] == 4 and st["failed"] == 0 and st["resident"] == 0
        assert st["atom_steps"] == sum(len(s["typ"]) * n for s, n in reqs)
        for k, x in enumerate(t):
            pos, vel, acc, box, rows = srv.result(x)
            _same(((pos, vel, acc, box), rows), alone[k])


@pytest.mark.gpu
def test_serving_springs_same_alone_and_in_mix():
    """A served run with spring pairs (the context switches to the spring
    variant of the pair kernels for every resident run) gives the same bits
    alone and beside runs without springs, and so do they."""
    spr = W.spring_alloy(6, 500.0, seed=45, quirk="fixed")  # 864 atoms, compute2
    spr["control"] = dict(spr["control"], out_steps=20)
    reqs = _requests()[:2] + [(spr, 120)]
    alone = [_alone_run(s, n) for s, n in reqs]
    with nd.Server(0, "mixed", hbm_budget=8e9, block_steps=40) as srv:
        t = [W.submit_to_server(srv, s, n) for s, n in reqs]
        for _ in range(40):
            srv.step()
            if all(srv.status(x) == 2 for x in t):
                break
        assert all(srv.status(x) == 2 for x in t)
        for k, x in enumerate(t):
            pos, vel, acc, box, rows = srv.result(x)
            _same(((pos, vel, acc, box), rows), alone[k])


@pytest.mark.gpu
def test_serving_admission_waits_for_budget():
    """With room for one run at a time the second is admitted only when the
    first retires; both results equal the runs alone."""
    reqs = _requests()[:2]
    alone = [_alone_run(s, n) for s, n in reqs]
    b = [_estimate(s) for s, _ in reqs]
    with nd.Server(0, "mixed", hbm_budget=max(b) + min(b) // 2, block_steps=50) as srv:
        t0 = W.submit_to_server(srv, reqs[0][0], reqs[0][1])
        t1 = W.submit_to_server(srv, reqs[1][0], reqs[1][1])
        srv.step()
        assert srv.status(t0) == 1 and srv.status(t1) == 0
        while srv.status(t0) != 2:
            srv.step()
        for _ in range(20):
            if srv.status(t1) == 2:
                break
            srv.step()
        assert srv.status(t1) == 2
        for k, x in enumerate((t0, t1)):
            pos, vel, acc, box, rows = srv.result(x)
            _same(((pos, vel, acc, box), rows), alone[k])


@pytest.mark.gpu
def test_serving_failed_run_leaves_others():
    """A run that cannot start (box narrower than two link cells) fails with
    its status; the run beside it completes."""
    good, n = _requests()[0]
    bad = W.cu_crystal(2, 300.0, seed=5, quirk="fixed")   # 7.2 A box < 2*(rc+skin)
    with nd.Server(0, "mixed", hbm_budget=8e9, block_steps=50) as srv:
        tg = W.submit_to_server(srv, good, n)
        tb = W.submit_to_server(srv, bad, 50)
        for _ in range(10):
            srv.step()
        assert srv.status(tb) == -5          # NDG_ERR_CELLS
        assert srv.status(tg) == 2
        with pytest.raises(nd.NdgError):
            srv.result(tb)
        pos, vel, acc, box, rows = srv.result(tg)
        _same(((pos, vel, acc, box), rows), _alone_run(good, n))

"""Bulk state transfer (ndg_load_state / ndg_get_state with sys = -1): every
live system moves in one call, in ascending id order, and the result is the
same bits as the per-system calls, before and after a run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

nd = pytest.importorskip("ndyn_omp_b200")
from ndyn_omp_b200 import workloads as W  # noqa: E402


def _specs():
    return [W.cu_crystal(5, 600.0, seed=21, quirk="fixed"),
            W.ar_liquid(6, 120.0, seed=22, quirk="fixed"),
            W.nacl_solid((4, 4, 4), 300.0, seed=23, quirk="fixed"),
            W.cu_crystal(7, 900.0, seed=24, quirk="fixed")]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_bulk_get_matches_per_system(prec):
    specs = _specs()
    with nd.Context(0, prec) as ctx:
        ids = [W.add_to_context(ctx, s) for s in specs]
        ctx.remove_system(ids[1])  # a hole in the id range: skipped
        live = [i for i in ids if i != ids[1]]
        ctx.run(30)
        pos, vel, acc, boxes = ctx.states()
        off = 0
        for k, i in enumerate(live):
            p, v, a, b = ctx.state(i)
            n = len(p)
            assert np.array_equal(pos[off:off + n], p)
            assert np.array_equal(vel[off:off + n], v)
            assert np.array_equal(acc[off:off + n], a)
            assert np.array_equal(boxes[k], b)
            off += n
        assert off == len(pos)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_bulk_load_matches_per_system(prec):
    specs = _specs()
    rng = np.random.default_rng(5)
    new = []
    for s in specs:
        n = len(s["typ"])
        new.append((W.jitter(s["pos"], s["box"], 0.03, rng), rng.normal(0, 0.01, (n, 3)),
                    rng.normal(0, 0.001, (n, 3)), np.asarray(s["box"]) * 1.01))
    out = []
    for bulk in (False, True):
        with nd.Context(0, prec) as ctx:
            ids = [W.add_to_context(ctx, s) for s in specs]
            ctx.run(10)
            if bulk:
                ctx.load_states(np.concatenate([q[0] for q in new]),
                                np.concatenate([q[1] for q in new]),
                                np.concatenate([q[2] for q in new]),
                                np.stack([q[3] for q in new]))
            else:
                for i, q in zip(ids, new):
                    ctx.load_state(i, *q)
            got = [ctx.state(i) for i in ids]
            for g, q in zip(got, new):
                assert np.array_equal(g[0], q[0]) and np.array_equal(g[1], q[1])
                assert np.array_equal(g[2], q[2]) and np.array_equal(g[3], q[3])
            rows = ctx.run(40)
            out.append(([ctx.state(i) for i in ids], rows))
    for a, b in zip(out[0][0], out[1][0]):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
    assert [(r["sys"], r["step"], r["pe"]) for r in out[0][1]] == \
        [(r["sys"], r["step"], r["pe"]) for r in out[1][1]]

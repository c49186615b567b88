"""GPU parity at the benchmark workloads' full sizes, against the CPU oracle
(all host threads), through the C ABI.

  * C2: LJ argon liquid, 256,000 atoms, NVT (fixed list semantics);
  * C3: rocksalt Buckingham solid, 1,048,576 atoms, NPT (thermostat and
    barostat);
  * a spread of the 512-replica ensemble (every 32nd replica, batched in one
    context as the benchmark runs them);
  * the two ensemble controls no workload above uses: total-energy control
    (mkIsoE, src/nd.f90:1159-1182) and a constant box velocity (BoxVel,
    src/nd.f90:178).

Bars, as in tests/test_gpu_parity.py:
  * link-cell assignment and neighbour pair multisets: bit-exact;
  * FP64 path: per-atom forces within 1e-12 relative L2, potential energy
    and virial within 1e-12; thermo rows of a run within 1e-11 (energy),
    1e-9 (kinetic energy, pressure) and 1e-12 (volume);
  * mixed path (FP32 pair math, 64-bit fixed-point sums): forces within the
    stated 1e-5 relative L2 force error, potential energy within 1e-6, the
    virial within 1e-5, thermo rows within 1e-6 (energies) and 1e-5
    (pressure).
"""
import os

import numpy as np
import pytest

from helpers import gpu_from_spec, oracle_from_spec, pair_multiset, rel_l2

pytestmark = pytest.mark.gpu

nd = pytest.importorskip("ndyn_omp_b200")
from ndyn_omp_b200 import workloads as W  # noqa: E402

THREADS = os.cpu_count()


def _oracle_lists(spec):
    o = oracle_from_spec(spec, threads=THREADS)
    assert o.setup_lists() == 0
    o.compute(1, 1)
    f, pe, vir, _ = o.forces()
    return o, dict(mcell=list(o.mcell()), cells=o.cells(), pairs=pair_multiset(o.neighbors()),
                   f=f, pe=pe, vir=vir)


def _check_lists_and_forces(spec, ref):
    errs = {}
    for prec, tol in (("fp64", 1e-12), ("mixed", 1e-5)):
        with nd.Context(0, prec) as ctx:
            sid = gpu_from_spec(ctx, spec)
            ctx.setup_lists()
            if prec == "fp64":
                assert list(ctx.mcell(sid)) == ref["mcell"]
                assert np.array_equal(ctx.cells(sid), ref["cells"]), "link-cell assignment"
                g = pair_multiset(ctx.neighbors(sid))
                assert len(g) == len(ref["pairs"])
                assert np.array_equal(g, ref["pairs"]), "neighbour pair multiset"
                del g
            ctx.compute0(True, True)
            f, pe, vir, _ = ctx.forces(sid)
        errs[prec] = rel_l2(f, ref["f"])
        assert errs[prec] < tol, (prec, errs[prec])
        pe_tol = 1e-12 if prec == "fp64" else 1e-6
        assert abs(pe - ref["pe"]) <= pe_tol * abs(ref["pe"]), (prec, pe, ref["pe"])
        assert rel_l2(vir, ref["vir"]) < tol, prec
    return errs


def _rows_match(rg, ro, prec):
    assert [r["step"] for r in rg] == [r["step"] for r in ro]
    e, k, p, v = (1e-11, 1e-9, 1e-9, 1e-12) if prec == "fp64" else (1e-6, 1e-6, 1e-5, 1e-6)
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=e), (prec, a["step"])
        assert a["ke"] == pytest.approx(b["ke"], rel=k), (prec, a["step"])
        # the pressure is a sum of terms of both signs: its tolerance is
        # relative to the size of the virial's diagonal
        scale = sum(abs(x) for x in b["virial"][:3]) / (3.0 * b["vol"])
        assert abs(a["press"] - b["press"]) <= p * scale + 1e-15, (prec, a["step"])
        assert a["vol"] == pytest.approx(b["vol"], rel=v), (prec, a["step"])


# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def c2():
    spec = W.ar_liquid(40, 120.0, seed=2, quirk="fixed")  # the bench's C2
    assert len(spec["typ"]) == 256000
    return spec


@pytest.fixture(scope="module")
def c3():
    spec = W.nacl_solid((64, 64, 32), 600.0, seed=3, quirk="fixed")  # the bench's C3
    assert len(spec["typ"]) == 1048576
    return spec


def test_c2_lists_and_forces(c2):
    _, ref = _oracle_lists(c2)
    errs = _check_lists_and_forces(c2, ref)
    print("C2 force error vs oracle:", errs)


def test_c3_lists_and_forces(c3):
    _, ref = _oracle_lists(c3)
    errs = _check_lists_and_forces(c3, ref)
    print("C3 force error vs oracle:", errs)


@pytest.mark.parametrize("cfg,nsteps", [("c2", 30), ("c3", 20)])
def test_config_runs(cfg, nsteps, c2, c3):
    """A short run of the workload, every fifth step written: the thermostat
    (C2) and thermostat plus barostat (C3) trajectories follow the oracle in
    both precisions."""
    spec = dict(c2 if cfg == "c2" else c3)
    spec["control"] = dict(spec["control"], out_steps=5)
    o = oracle_from_spec(spec, threads=THREADS)
    rc, ro = o.run(nsteps, spec["control"]["dt"])
    assert rc == 0
    _, _, _, bo = o.state()
    for prec in ("fp64", "mixed"):
        with nd.Context(0, prec) as ctx:
            sid = gpu_from_spec(ctx, spec)
            rg = ctx.run(nsteps)
            _, _, _, bg = ctx.state(sid)
            nup = ctx.list_updates(sid)
        _rows_match(rg, ro, prec)
        assert np.allclose(bg, bo, rtol=1e-12 if prec == "fp64" else 1e-6, atol=0)
        if prec == "fp64":
            assert nup == o.list_updates


# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def replica_sample():
    specs = W.replica_ensemble(512, seed=4, quirk="fixed")  # the bench's c4
    rng = np.random.default_rng(77)
    out = []
    for k in range(0, 512, 32):
        sp = dict(specs[k])
        # the crystals start on their lattice (zero net force): a small
        # displacement makes the force comparison meaningful
        sp["pos"] = W.jitter(sp["pos"], sp["box"], 0.05, rng)
        sp["control"] = dict(sp["control"], out_steps=10)
        out.append(sp)
    return out


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_replica_sample_forces(replica_sample, prec, tol):
    refs = []
    for sp in replica_sample:
        o = oracle_from_spec(sp, threads=THREADS)
        assert o.setup_lists() == 0
        o.compute(1, 1)
        refs.append(o.forces())
    with nd.Context(0, prec) as ctx:
        ids = [gpu_from_spec(ctx, sp) for sp in replica_sample]
        ctx.setup_lists()
        ctx.compute0(True, True)
        got = [ctx.forces(i) for i in ids]
    for (fg, peg, virg, _), (fo, peo, viro, _) in zip(got, refs):
        assert rel_l2(fg, fo) < tol
        assert abs(peg - peo) <= (1e-12 if prec == "fp64" else 1e-6) * abs(peo)
        assert rel_l2(virg, viro) < tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_replica_sample_batched_run(replica_sample, prec):
    """The sampled replicas stepped together in one context, each with its own
    thermostat, follow their oracle runs one by one."""
    nsteps = 40
    ro = []
    for sp in replica_sample:
        o = oracle_from_spec(sp, threads=THREADS)
        rc, rows = o.run(nsteps, sp["control"]["dt"])
        assert rc == 0
        ro.append((rows, o.list_updates))
    with nd.Context(0, prec) as ctx:
        ids = [gpu_from_spec(ctx, sp) for sp in replica_sample]
        rows = ctx.run(nsteps)
        nup = [ctx.list_updates(i) for i in ids]
    for k, i in enumerate(ids):
        _rows_match([r for r in rows if r["sys"] == i], ro[k][0], prec)
        if prec == "fp64":
            assert nup[k] == ro[k][1]


# ---------------------------------------------------------------------------
def test_run_isoenergetic_fp64():
    """Total-energy control (Isoenergetic; mkIsoE after every step): velocity
    scale 1 - dt/Eparm*(e0/(PE+KE) - 1), src/nd.f90:1159-1182."""
    spec = W.cu_crystal(6, 900.0, seed=51, quirk="fixed")
    spec["pos"] = W.jitter(spec["pos"], spec["box"], 0.05, np.random.default_rng(52))
    spec["control"] = dict(spec["control"], out_steps=10, isoenergetic=1, e_freq=1, e_parm=2.0)
    o = oracle_from_spec(spec, threads=THREADS)
    rc, ro = o.run(100, spec["control"]["dt"])
    assert rc == 0
    po, vo, _, _ = o.state()
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        rg = ctx.run(100)
        pg, vg, _, _ = ctx.state(sid)
    _rows_match(rg, ro, "fp64")
    for a, b in zip(rg, ro):
        assert abs(a["eerr"] - b["eerr"]) <= 1e-10
    assert rel_l2(pg, po) < 1e-12
    assert rel_l2(vg, vo) < 1e-10


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_run_box_velocity(prec):
    """A constant box velocity (BoxLoad/BoxVel: box = box + boxVel*dt after
    every step, src/nd.f90:178) with the fixed rebuild test, which rebuilds
    the lists as the box shrinks along one axis."""
    spec = W.ar_liquid(8, 120.0, seed=53, quirk="fixed")
    spec["control"] = dict(spec["control"], out_steps=10, box_load=1,
                           box_vel=[0.02, -0.03, 0.0])
    o = oracle_from_spec(spec, threads=THREADS)
    rc, ro = o.run(120, spec["control"]["dt"])
    assert rc == 0
    _, _, _, bo = o.state()
    with nd.Context(0, prec) as ctx:
        sid = gpu_from_spec(ctx, spec)
        rg = ctx.run(120)
        _, _, _, bg = ctx.state(sid)
        nup = ctx.list_updates(sid)
    _rows_match(rg, ro, prec)
    assert np.array_equal(bg, bo)  # the same FP64 additions on both sides
    assert ro[-1]["vol"] != ro[0]["vol"]
    if prec == "fp64":
        assert nup == o.list_updates

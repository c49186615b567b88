"""GPU parity: the CUDA library (through its C ABI) against the CPU oracle on
identical seeded inputs.

Bars (stated per test):
  * link-cell assignment and neighbour pairs: bit-exact (cells equal, pair
    multisets equal, both in the reference semantics and the fixed one);
  * FP64 path: per-atom forces within 1e-12 relative L2 of the oracle
    (only the summation order differs), PE/virial within 1e-12;
  * mixed path: forces within 1e-5 relative L2 (the stated force error),
    PE within 1e-6, virial within 1e-5;
  * integrate1 bit-exact; full runs follow the oracle's thermo rows.
"""
import numpy as np
import pytest

from helpers import gpu_from_spec, oracle_from_spec, pair_multiset, rel_l2

pytestmark = pytest.mark.gpu

nd = pytest.importorskip("ndyn_omp_b200")
from ndyn_omp_b200 import workloads as W  # noqa: E402


def small_specs():
    return {
        "cu_ref": W.cu_crystal(8, 300.0, seed=11, quirk="ref"),          # 2048 atoms, M=4
        "ar_fixed": W.ar_liquid(6, 120.0, seed=12, quirk="fixed"),        # 864 atoms, M=3
        "nacl_fixed": W.nacl_solid((6, 6, 6), 600.0, seed=13, quirk="fixed"),  # 1728 atoms
        "cu_m2_ref": W.cu_crystal(5, 900.0, seed=14, quirk="ref"),        # 500 atoms, M=2
        "cu_m2_fixed": W.cu_crystal(5, 900.0, seed=14, quirk="fixed"),
        "cu_m6_ref": W.cu_crystal(12, 600.0, seed=15, quirk="ref"),      # 6912 atoms, M=6
        # two types, one one-sided (asym) pair: compute1's rules
        "alloy_fixed": W.onesided_alloy(8, 300.0, seed=16, quirk="fixed"),  # 2048 atoms, M=4
    }


def _jitter(spec, amp, seed):
    rng = np.random.default_rng(seed)
    spec = dict(spec)
    spec["pos"] = W.jitter(spec["pos"], spec["box"], amp, rng)
    return spec


@pytest.fixture(scope="module")
def specs():
    s = small_specs()
    s["cu_ref"] = _jitter(s["cu_ref"], 0.05, 99)
    s["cu_m6_ref"] = _jitter(s["cu_m6_ref"], 0.1, 98)
    s["alloy_fixed"] = _jitter(s["alloy_fixed"], 0.05, 97)
    return s


@pytest.mark.parametrize("name", ["cu_ref", "ar_fixed", "nacl_fixed", "cu_m2_ref", "cu_m2_fixed",
                                  "cu_m6_ref", "alloy_fixed"])
def test_cells_and_neighbour_pairs_bit_exact(specs, name):
    spec = specs[name]
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        assert list(ctx.mcell(sid)) == list(o.mcell())
        assert np.array_equal(ctx.cells(sid), o.cells()), "link-cell assignment differs"
        g = pair_multiset(ctx.neighbors(sid))
        r = pair_multiset(o.neighbors())
        assert len(g) == len(r)
        assert np.array_equal(g, r), "neighbour pair multiset differs"
    if name == "cu_m2_ref":
        # 2 link cells per direction: the reference stencil repeats pairs
        assert len(r) > len(np.unique(r))
    if name == "cu_m2_fixed":
        assert len(r) == len(np.unique(r))


@pytest.mark.parametrize("name", ["cu_ref", "ar_fixed", "nacl_fixed", "cu_m2_ref"])
def test_compute0_fp64(specs, name):
    spec = specs[name]
    o = oracle_from_spec(spec)
    o.setup_lists()
    o.compute0(1, 1)
    fo, peo, viro, _ = o.forces()
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        ctx.compute0(True, True)
        fg, peg, virg, _ = ctx.forces(sid)
    assert rel_l2(fg, fo) < 1e-12
    assert abs(peg - peo) <= 1e-12 * abs(peo)
    assert rel_l2(virg, viro) < 1e-12


@pytest.mark.parametrize("name", ["cu_ref", "ar_fixed", "nacl_fixed"])
def test_compute0_mixed_force_error(specs, name):
    """Mixed precision: FP32 pair math + 64-bit fixed-point sums; the
    stated bar is 1e-5 relative L2 force error against the FP64 oracle."""
    spec = specs[name]
    o = oracle_from_spec(spec)
    o.setup_lists()
    o.compute0(1, 1)
    fo, peo, viro, _ = o.forces()
    with nd.Context(0, "mixed") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        ctx.compute0(True, True)
        fg, peg, virg, _ = ctx.forces(sid)
    err = rel_l2(fg, fo)
    assert err < 1e-5, err
    assert abs(peg - peo) <= 1e-6 * abs(peo)
    assert rel_l2(virg, viro) < 1e-5


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_onesided_pairs_compute1(specs, prec, tol):
    """A one-sided (asym) pair: forces follow compute1 (src/nd.f90:364-530),
    only symmetric pairs add energy and virial; same bars as compute0."""
    spec = specs["alloy_fixed"]
    o = oracle_from_spec(spec)
    o.setup_lists()
    o.compute(1, 1)
    fo, peo, viro, _ = o.forces()
    with nd.Context(0, prec) as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        ctx.compute0(True, True)
        fg, peg, virg, _ = ctx.forces(sid)
    assert rel_l2(fg, fo) < tol
    assert abs(peg - peo) <= (1e-12 if prec == "fp64" else 1e-6) * abs(peo)
    assert rel_l2(virg, viro) < tol
    assert np.linalg.norm(fo.sum(axis=0)) > 1e-6 * np.abs(fo).sum()  # no Newton-3 balance


def _spring_spec(onesided, seed):
    spec = W.spring_alloy(6, 300.0, seed=seed, quirk="fixed", onesided=onesided)  # 864 atoms
    ipos = np.asarray(spec["pos"], np.float64).reshape(-1, 3).copy()
    spec["pos"] = W.jitter(spec["pos"], spec["box"], 0.08, np.random.default_rng(seed + 1))
    return spec, ipos


@pytest.mark.parametrize("onesided", [False, True])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_springs_compute2_compute3(onesided, prec, tol):
    """Spring pairs (compute2; compute3 with a one-sided line) strained
    against the lattice: forces, energy and virial against the oracle."""
    spec, ipos = _spring_spec(onesided, 20)
    o = oracle_from_spec(spec)
    o.init_positions(ipos)
    o.setup_lists()
    o.compute(1, 1)
    fo, peo, viro, _ = o.forces()
    with nd.Context(0, prec) as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.set_initial_positions(sid, ipos)
        ctx.setup_lists()
        assert np.array_equal(pair_multiset(ctx.neighbors(sid)), pair_multiset(o.neighbors()))
        ctx.compute0(True, True)
        fg, peg, virg, _ = ctx.forces(sid)
    assert rel_l2(fg, fo) < tol
    assert abs(peg - peo) <= (1e-12 if prec == "fp64" else 1e-6) * abs(peo)
    assert rel_l2(virg, viro) < tol


def test_run_springs_fp64():
    """A run with springs: the prologue takes the starting positions as the
    initial configuration (src/nd.f90:104) on both sides."""
    spec = W.spring_alloy(6, 600.0, seed=22, quirk="fixed")
    spec["control"] = dict(spec["control"], out_steps=10)
    o, ro, rg, (pg, _, _, _), nup = _run_both(spec, 80)
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-10, abs=1e-9)
        assert a["ke"] == pytest.approx(b["ke"], rel=1e-9)
    po, _, _, _ = o.state()
    assert rel_l2(pg, po) < 1e-12
    assert nup == o.list_updates


def test_integrate1_bit_exact(specs):
    spec = dict(specs["ar_fixed"])
    rng = np.random.default_rng(5)
    spec["acc"] = rng.standard_normal(spec["pos"].shape) * 1e-3
    o = oracle_from_spec(spec)
    o.setup_lists()
    o.integrate1()
    po, _, _, _ = o.state()
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        ctx.integrate1()
        pg, _, _, _ = ctx.state(sid)
    assert np.array_equal(pg, po)


def test_routines_step_by_step_match_oracle(specs):
    """integrate1 -> compute0 -> integrate2 -> mkIsoKE -> mkIsoP called one
    by one through the ABI, as dynamics calls them."""
    spec = dict(specs["nacl_fixed"])
    o = oracle_from_spec(spec)
    o.setup_lists()
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        for _ in range(3):
            o.check_list_update()
            ctx.check_list_update()
            o.integrate1()
            ctx.integrate1()
            o.compute0(1, 1)
            ctx.compute0(True, True)
            o.integrate2(1)
            ctx.integrate2(True)
            o.L.ora_mk_iso_ke(o.s)
            ctx.mk_iso_ke(sid)
            o.L.ora_mk_iso_p(o.s)
            ctx.mk_iso_p(sid)
        po, vo, ao, bo = o.state()
        pg, vg, ag, bg = ctx.state(sid)
        _, peo, viro, keo = o.forces()
        _, peg, virg, keg = ctx.forces(sid)
    assert rel_l2(pg, po) < 1e-13
    assert rel_l2(vg, vo) < 1e-10
    assert rel_l2(bg, bo) < 1e-13
    assert abs(keg - keo) <= 1e-10 * abs(keo)
    assert abs(peg - peo) <= 1e-12 * abs(peo)


def _run_both(spec, nsteps, precision="fp64", threads=None):
    o = oracle_from_spec(spec, threads=threads)
    rc, rows_o = o.run(nsteps, spec["control"]["dt"])
    assert rc == 0
    with nd.Context(0, precision) as ctx:
        sid = gpu_from_spec(ctx, spec)
        rows_g = ctx.run(nsteps)
        st = ctx.state(sid)
        nup = ctx.list_updates(sid)
    return o, rows_o, rows_g, st, nup


def test_run_nve_crystal_fp64(specs):
    spec = specs["cu_ref"]
    spec = dict(spec)
    spec["control"] = dict(spec["control"], out_steps=10)
    o, ro, rg, (pg, vg, _, _), nup = _run_both(spec, 100)
    assert [r["step"] for r in rg] == [r["step"] for r in ro]
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-11)
        assert a["ke"] == pytest.approx(b["ke"], rel=1e-9)
        assert a["press"] == pytest.approx(b["press"], rel=1e-9, abs=1e-12)
        assert a["vol"] == b["vol"]
    po, vo, _, _ = o.state()
    assert rel_l2(pg, po) < 1e-12
    assert nup == o.list_updates


def test_run_onesided_fp64(specs):
    """Dynamics with a one-sided pair: the run takes compute1 on both sides."""
    spec = dict(specs["alloy_fixed"])
    spec["control"] = dict(spec["control"], out_steps=10)
    o, ro, rg, (pg, _, _, _), nup = _run_both(spec, 100)
    assert [r["step"] for r in rg] == [r["step"] for r in ro]
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-11)
        assert a["ke"] == pytest.approx(b["ke"], rel=1e-9)
    po, _, _, _ = o.state()
    assert rel_l2(pg, po) < 1e-12
    assert nup == o.list_updates


def _holds(spec):
    """Two hold groups: the atoms with z in the lower quarter move by a fixed
    x/z displacement per step, one type is held with no constrained axis."""
    pos = np.asarray(spec["pos"], np.float64).reshape(-1, 3)
    hold = np.zeros(len(pos), np.int32)
    hold[pos[:, 2].astype(np.float32) <= np.float32(-0.25)] = 1
    hold[(hold == 0) & (np.asarray(spec["typ"]) == 2)] = 2
    return hold, [[True, False, True], [False, False, False]], [[2e-5, 0.0, -1e-5], [0, 0, 0]]


@pytest.mark.parametrize("name", ["alloy_fixed", "cu_ref"])
def test_run_hold_groups_fp64(specs, name):
    """Hold groups with displacement conditions (integrate1's Nhold branch,
    src/nd.f90:1048-1077) follow the oracle through a run."""
    spec = dict(specs[name])
    spec["control"] = dict(spec["control"], out_steps=10)
    hold, dirs, du = _holds(spec)
    o = oracle_from_spec(spec)
    o.set_holds(hold, dirs, du)
    rc, ro = o.run(60, spec["control"]["dt"])
    assert rc == 0
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.set_holds(sid, hold, dirs, du)
        rg = ctx.run(60)
        pg, _, _, _ = ctx.state(sid)
    po, _, _, _ = o.state()
    assert rel_l2(pg, po) < 1e-12
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-11)
        assert a["ke"] == pytest.approx(b["ke"], rel=1e-9)
    p0 = np.asarray(spec["pos"], np.float64).reshape(-1, 3)
    g1 = hold == 1
    assert np.allclose(pg[g1, 0] - p0[g1, 0], 60 * 2e-5, rtol=0, atol=1e-13)  # 60 roundings


def test_run_nvt_liquid_fixed_rebuilds(specs):
    """LJ liquid with the fixed rebuild criterion: lists are rebuilt on the
    same steps as the oracle and the thermostat trajectory follows it."""
    spec = dict(specs["ar_fixed"])
    spec["control"] = dict(spec["control"], out_steps=20)
    o, ro, rg, _, nup = _run_both(spec, 200)
    assert nup == o.list_updates and nup > 0
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-8)
        assert a["ke"] == pytest.approx(b["ke"], rel=1e-8)


def test_run_npt_barostat(specs):
    spec = dict(specs["nacl_fixed"])
    spec["control"] = dict(spec["control"], out_steps=25)
    o, ro, rg, (_, _, _, box), _ = _run_both(spec, 100)
    _, _, _, bo = o.state()
    assert np.allclose(box, bo, rtol=1e-12)
    for a, b in zip(rg, ro):
        assert a["vol"] == pytest.approx(b["vol"], rel=1e-12)
        assert a["press"] == pytest.approx(b["press"], rel=1e-8, abs=1e-12)


def test_run_skin0_rebuilds_every_step():
    """Reference semantics with skin 0: CheckListUpdate fires every step
    (examples/testCAF/OMP_4/out reports 98 updates in 100 steps)."""
    spec = W.cu_crystal(6, 300.0, seed=21, quirk="ref")
    spec["control"] = dict(spec["control"], skin=0.0, out_steps=10)
    o, ro, rg, _, nup = _run_both(spec, 30)
    assert nup == o.list_updates
    assert nup >= 28
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-11)


def test_batch_equals_alone(specs):
    """Several systems in one context (one launch per kernel) give bitwise
    the same trajectories as each system alone."""
    names = ["cu_ref", "ar_fixed", "nacl_fixed", "cu_m2_ref"]
    alone = {}
    for n in names:
        with nd.Context(0, "mixed") as ctx:
            sid = gpu_from_spec(ctx, specs[n])
            ctx.run(50)
            alone[n] = ctx.state(sid)
    with nd.Context(0, "mixed") as ctx:
        ids = {n: gpu_from_spec(ctx, specs[n]) for n in names}
        ctx.run(50)
        for n in names:
            got = ctx.state(ids[n])
            for a, b in zip(got, alone[n]):
                assert np.array_equal(a, b), n


def test_many_systems_round_robin_build():
    """300 systems in one context: the prologue build deals their tiles
    round-robin (a list of 256 or more systems), a step's few rebuilds take
    them from the build's work counter; either way each system's lists and
    trajectory are the same bits as alone."""
    rng = np.random.default_rng(40)
    many = [W.cu_crystal(5, float(T), seed=int(100 + k), quirk="fixed")
            for k, T in enumerate(rng.uniform(300.0, 1500.0, 300))]
    sample = [0, 137, 299]
    alone = {}
    for k in sample:
        with nd.Context(0, "mixed") as ctx:
            sid = gpu_from_spec(ctx, many[k])
            ctx.setup_lists()
            nb = pair_multiset(ctx.neighbors(sid))
            ctx.run(40)
            alone[k] = (nb, ctx.state(sid), ctx.list_updates(sid))
    with nd.Context(0, "mixed") as ctx:
        ids = [gpu_from_spec(ctx, sp) for sp in many]
        ctx.setup_lists()
        for k in sample:
            assert np.array_equal(pair_multiset(ctx.neighbors(ids[k])), alone[k][0])
        ctx.run(40)
        for k in sample:
            for a, b in zip(ctx.state(ids[k]), alone[k][1]):
                assert np.array_equal(a, b), k
            assert ctx.list_updates(ids[k]) == alone[k][2]
        assert sum(ctx.list_updates(i) for i in ids) > 0  # some steps rebuilt


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_run_continue_equals_one_run(specs, prec):
    """ndg_run(n) then ndg_run_continue(m) is the same run as ndg_run(n + m):
    the same states and write_thermo records (e0 and the step counter carry
    on), which lets a caller stop every ConfOutFreq steps to write the
    model."""
    spec = dict(specs["nacl_fixed"])
    spec["control"] = dict(spec["control"], out_steps=7)
    out = []
    for pieces in ((60,), (25, 10, 25)):
        with nd.Context(0, prec) as ctx:
            sid = gpu_from_spec(ctx, spec)
            rows = ctx.run(pieces[0])
            for m in pieces[1:]:
                rows += ctx.run(m, cont=True)
            out.append((ctx.state(sid), rows, ctx.list_updates(sid)))
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    assert out[0][1] == out[1][1]
    assert out[0][2] == out[1][2]


@pytest.mark.parametrize("quirk", ["ref", "fixed"])
def test_cell_build_equals_tile_build(quirk):
    """The list build's two forms give every atom the same list in the same
    order.  400 systems with 2, 3, 4 and 5 link cells per axis (22,400 cells)
    take the cell form in their shared prologue; each alone takes the tile
    form.  The sampled systems' pair multisets are equal, and so are their
    mixed-precision states after a short run, whose fixed-point sums follow
    the list order."""
    rng = np.random.default_rng(81)
    makers = [lambda k: W.cu_crystal(5, 900.0, seed=1000 + k, quirk=quirk),   # 2 cells per axis
              lambda k: W.cu_crystal(6, 600.0, seed=2000 + k, quirk=quirk),   # 3
              lambda k: W.cu_crystal(8, 300.0, seed=3000 + k, quirk=quirk),   # 4
              lambda k: W.ar_liquid(9, 120.0, seed=4000 + k, quirk=quirk)]    # 5
    many = []
    for k in range(100):
        for mk in makers:
            sp = mk(k)
            sp["pos"] = W.jitter(sp["pos"], sp["box"], 0.05, rng)
            # the reference's own NeiMax estimate does not allow for the
            # repeated cells of a 2-cell grid: a caller's NeiMax does
            sp["control"] = dict(sp["control"], neimax=300)
            many.append(sp)
    sample = [0, 1, 2, 3, 201, 398, 399]
    alone = {}
    for k in sample:
        with nd.Context(0, "mixed") as ctx:
            sid = gpu_from_spec(ctx, many[k])
            ctx.setup_lists()
            alone[k] = (pair_multiset(ctx.neighbors(sid)), None)
            ctx.run(5)
            alone[k] = (alone[k][0], ctx.state(sid))
    with nd.Context(0, "mixed") as ctx:
        ids = [gpu_from_spec(ctx, sp) for sp in many]
        ctx.setup_lists()
        for k in sample:
            assert np.array_equal(pair_multiset(ctx.neighbors(ids[k])), alone[k][0]), k
        ctx.run(5)
        for k in sample:
            for a, b in zip(ctx.state(ids[k]), alone[k][1]):
                assert np.array_equal(a, b), k


def test_deterministic_repeat(specs):
    out = []
    for _ in range(2):
        with nd.Context(0, "fp64") as ctx:
            sid = gpu_from_spec(ctx, specs["ar_fixed"])
            rows = ctx.run(60)
            out.append((ctx.state(sid), rows))
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    assert out[0][1] == out[1][1]


@pytest.fixture(scope="module")
def large_liquid():
    # 78,732 atoms = 616 tiles of 128: every persistent CTA of the pair kernel
    # works through several tiles (and table staging) per launch
    return W.ar_liquid(27, 120.0, seed=31, quirk="fixed")


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
def test_large_system_forces(large_liquid, prec, tol):
    o = oracle_from_spec(large_liquid)
    o.setup_lists()
    o.compute0(1, 1)
    fo, peo, viro, _ = o.forces()
    with nd.Context(0, prec) as ctx:
        sid = gpu_from_spec(ctx, large_liquid)
        ctx.setup_lists()
        ctx.compute0(True, True)
        fg, peg, virg, _ = ctx.forces(sid)
        assert np.array_equal(pair_multiset(ctx.neighbors(sid)), pair_multiset(o.neighbors()))
    assert rel_l2(fg, fo) < tol
    assert abs(peg - peo) <= max(tol, 1e-6) * abs(peo)


def test_large_system_run_follows_oracle(large_liquid):
    spec = dict(large_liquid)
    spec["control"] = dict(spec["control"], out_steps=10)
    o, ro, rg, _, nup = _run_both(spec, 40, precision="mixed")
    assert nup == o.list_updates
    for a, b in zip(rg, ro):
        assert a["pe"] == pytest.approx(b["pe"], rel=1e-6)
        assert a["ke"] == pytest.approx(b["ke"], rel=1e-5)


@pytest.mark.parametrize("quirk", ["ref", "fixed"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-5)])
def test_cutoff_shell_decided_like_the_oracle(prec, tol, quirk):
    """Pairs on the cutoff: an FCC Morse lattice stretched so that its fourth
    neighbour shell (12 atoms at a*sqrt(2)) lies at the 6.0 A cutoff, the
    atoms displaced by at most 1e-7 A.  Every such pair's FP32 squared
    distance is within the mixed loop's 1e-5 band, so the reference's FP64
    test (compute0, src/nd.f90:283-296) must decide it, in the full chunks'
    f32x2 path and in the masked tail alike (54 list entries per atom).  A
    pair decided the other way would move two forces by the Morse force at
    the cutoff, ~1.3e-2 eV/A; the bar is 1e-5 eV/A (1e-10 in FP64)."""
    rng = np.random.default_rng(31)
    a = 6.0 / np.sqrt(2.0)
    pos, box = W.lattice((6, 6, 6), a, W.FCC_BASIS)
    pos = W.jitter(pos, box, 1e-7, rng)
    n = len(pos)
    spec = dict(masses=W.CU_MORSE["masses"], pairs=W.CU_MORSE["pairs"],
                typ=np.ones(n, np.int32), pos=pos, box=box, vel=np.zeros((n, 3)),
                control=dict(dt=0.1, skin=0.5, out_steps=100, quirk=quirk))
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0
    o.compute(1, 1)
    fo, peo, _, _ = o.forces()
    with nd.Context(0, prec) as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        assert ctx.neighbor_count(sid) == 54 * n  # shells 1-4 within rcut + skin
        ctx.compute0(True, True)
        fg, peg, _, _ = ctx.forces(sid)
    assert np.max(np.abs(np.asarray(fg) - np.asarray(fo))) < tol
    assert abs(peg - peo) <= (1e-12 if prec == "fp64" else 1e-7) * abs(peo)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_list_split_by_length(specs, prec):
    """Atoms to threads by list length: a context of an Ar liquid (~70
    entries per atom), a Cu crystal (~90) and a rocksalt solid (~130), its
    long-list systems in launches of their own with 2 or 4 threads per atom.
    Mixed precision: the same bits as one class (the fixed-point chunk sums
    do not depend on the threads); FP64: within the summation-order bar."""
    systems = [specs["ar_fixed"], specs["cu_ref"], specs["nacl_fixed"]]
    out = []
    for split, tl in ((0, 2), (100, 2), (100, 4)):
        with nd.Context(0, prec) as ctx:
            ids = [gpu_from_spec(ctx, sp) for sp in systems]
            ctx.set_tuning(1, 100)
            ctx.set_list_split(split, tl)
            assert ctx.list_split() == (split, tl)
            rows = ctx.run(40)
            out.append(([ctx.state(i) for i in ids], rows))
    for k in (1, 2):
        for sa, sb in zip(out[0][0], out[k][0]):
            for a, b in zip(sa, sb):
                if prec == "mixed":
                    assert np.array_equal(a, b)
                else:
                    assert np.allclose(a, b, rtol=1e-9, atol=1e-11)
        if prec == "mixed":
            assert out[0][1] == out[k][1]
        else:
            for ra, rb in zip(out[0][1], out[k][1]):
                assert ra["pe"] == pytest.approx(rb["pe"], rel=1e-10)


def test_autotune_split_restores_state(specs):
    """The autotuner's list-length trials leave no trace either (systems of
    mean list lengths 1.5x apart), and the split it keeps, if any, changes no
    bit of a mixed run."""
    systems = [specs["ar_fixed"], specs["nacl_fixed"]]
    res = []
    for tune in (False, True):
        with nd.Context(0, "mixed") as ctx:
            ids = [gpu_from_spec(ctx, sp) for sp in systems]
            ctx.run(20)
            before = [ctx.state(i) for i in ids]
            if tune:
                ctx.autotune(10)
                for i, b in zip(ids, before):
                    for x, y in zip(ctx.state(i), b):
                        assert np.array_equal(x, y)
                r, t = ctx.list_split()
                assert r >= 0 and t in (1, 2, 4, 8)
            res.append(([ctx.state(i) for i in ids], ctx.run(30, cont=True)))
    for sa, sb in zip(res[0][0], res[1][0]):
        for a, b in zip(sa, sb):
            assert np.array_equal(a, b)
    assert res[0][1] == res[1][1]


def test_autotune_restores_state(specs):
    """The autotuner's trial steps leave no trace: the state after tuning
    equals the state before it, and a continued run equals one without
    tuning (mixed precision: fixed-point sums make every launch shape give
    the same bits)."""
    spec = specs["ar_fixed"]
    res = []
    for tune in (False, True):
        with nd.Context(0, "mixed") as ctx:
            sid = gpu_from_spec(ctx, spec)
            ctx.run(20)
            before = ctx.state(sid)
            nup = ctx.list_updates(sid)
            if tune:
                ctx.autotune(10)
                for a, b in zip(before, ctx.state(sid)):
                    assert np.array_equal(a, b)
                assert ctx.list_updates(sid) == nup
            rows = ctx.run(30, cont=True)
            res.append((ctx.state(sid), rows, ctx.list_updates(sid)))
    for a, b in zip(res[0][0], res[1][0]):
        assert np.array_equal(a, b)
    assert res[0][1] == res[1][1]
    assert res[0][2] == res[1][2]


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-10), ("mixed", 1e-6)])
def test_autotune_skin(prec, tol):
    """The rebuild-interval autotuner undoes its trial (the state is the same
    bits afterwards), leaves reference-semantics systems' skins alone, keeps
    the others within [0.5, 2] x their skin, and changes no physics: a run
    after tuning follows an untuned run within the precision's tolerance
    (only the list lengths and orders differ)."""
    systems = [W.cu_crystal(7, 1500.0, seed=61, quirk="fixed"),
               W.ar_liquid(7, 120.0, seed=62, quirk="fixed"),
               W.cu_crystal(8, 100.0, seed=63, quirk="fixed"),
               W.cu_crystal(6, 900.0, seed=64, quirk="ref")]
    for sp in systems:
        sp["control"] = dict(sp["control"], out_steps=10)
    runs = []
    for tune in (False, True):
        with nd.Context(0, prec) as ctx:
            ids = [gpu_from_spec(ctx, sp) for sp in systems]
            ctx.run(20)
            skins0 = [ctx.control(i).skin for i in ids]
            if tune:
                before = [ctx.state(i) for i in ids]
                changed = ctx.autotune_skin(40)
                for i, b in zip(ids, before):
                    for x, y in zip(ctx.state(i), b):
                        assert np.array_equal(x, y)
                skins = [ctx.control(i).skin for i in ids]
                assert skins[3] == skins0[3]  # reference semantics: untouched
                for a, b in zip(skins, skins0):
                    assert 0.5 * b - 1e-12 <= a <= 2.0 * b + 1e-12
                assert changed == sum(a != b for a, b in zip(skins, skins0))
            rows = ctx.run(60, cont=True)
            runs.append(rows)
    assert [(r["sys"], r["step"]) for r in runs[0]] == [(r["sys"], r["step"]) for r in runs[1]]
    for a, b in zip(runs[0], runs[1]):
        assert a["pe"] == pytest.approx(b["pe"], rel=tol)
        assert a["ke"] == pytest.approx(b["ke"], rel=tol)


@pytest.mark.parametrize("quirk", ["ref", "fixed"])
def test_direct_build_coarse_cells(quirk):
    """A 12 A list radius on a 36 A box: a 3x3x3 cell grid, ~4000 candidates
    per tile and lists of ~800, beyond the staged build's shared buffers.
    The direct build path must give the same cells, pairs and forces."""
    spec = W.cu_crystal(10, 300.0, seed=51, quirk=quirk)
    spec = _jitter(spec, 0.05, 52)
    spec["control"] = dict(spec["control"], skin=6.0)
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0
    o.compute0(1, 1)
    fo, peo, _, _ = o.forces()
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        assert list(ctx.mcell(sid)) == [3, 3, 3]
        assert np.array_equal(ctx.cells(sid), o.cells())
        assert np.array_equal(pair_multiset(ctx.neighbors(sid)), pair_multiset(o.neighbors()))
        ctx.compute0(True, True)
        fg, peg, _, _ = ctx.forces(sid)
    assert rel_l2(fg, fo) < 1e-12
    assert abs(peg - peo) <= 1e-12 * abs(peo)


def test_nve_drift_1000_steps_fp64_and_mixed():
    """C1 (Cu 10^3 cells, Morse, 300 K, NVE, reference semantics), 1000 steps
    in the oracle, the FP64 path and the mixed path.  Stated tolerances on
    the energy error (PE+KE-e0)/e0 at every write_thermo row: FP64 within
    1e-8 absolute of the oracle (summation order only; the trajectories
    separate slowly), mixed within 1e-7 absolute, and the mixed drift over
    steps 100..1000 within 1e-8 of the FP64 drift."""
    spec = W.cu_crystal(10, 300.0, seed=1, quirk="ref")
    spec["control"] = dict(spec["control"], out_steps=100)
    o = oracle_from_spec(spec)
    rc, ro = o.run(1000, spec["control"]["dt"])
    assert rc == 0
    res = {}
    for p in ("fp64", "mixed"):
        with nd.Context(0, p) as ctx:
            gpu_from_spec(ctx, spec)
            res[p] = ctx.run(1000)
    g, m = res["fp64"], res["mixed"]
    assert len(ro) == len(g) == len(m) == 11
    for a, b, c in zip(ro, g, m):
        assert a["step"] == b["step"] == c["step"]
        assert abs(b["eerr"] - a["eerr"]) <= 1e-8
        assert abs(c["eerr"] - a["eerr"]) <= 1e-7
        assert c["pe"] == pytest.approx(a["pe"], rel=1e-7)
    drift_g = g[-1]["eerr"] - g[1]["eerr"]
    drift_m = m[-1]["eerr"] - m[1]["eerr"]
    assert abs(drift_m - drift_g) <= 1e-8


def test_gather_depth_same_bits(specs):
    """The mixed loop's gather depth (4 or 8 neighbour loads in flight) is a
    pure launch choice: the same chunks are summed in the same order, so
    forces and trajectories are the same bits."""
    spec = specs["ar_fixed"]
    out = []
    for depth in (4, 8):
        with nd.Context(0, "mixed") as ctx:
            sid = gpu_from_spec(ctx, spec)
            ctx.set_tuning(1, 100)
            ctx.set_gather_depth(depth)
            assert ctx.gather_depth() == depth
            rows = ctx.run(40)
            out.append((ctx.state(sid), rows))
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    assert out[0][1] == out[1][1]

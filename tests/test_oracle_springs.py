"""The oracle's compute2/compute3 (src/nd.f90:531-933): 'spring' pairs act
through their strain against the initial configuration.  Pinned on the CPU
against an all-pairs numpy evaluation of the same rules (within 1e-12; only
the summation order differs), for compute2 (all pairs symmetric) and
compute3 (a one-sided LJ line); a spring network at its initial
configuration carries no force."""
import numpy as np
import pytest

from helpers import oracle_from_spec, rel_l2
from ndyn_omp_b200 import workloads as W


def _brute(o, spec, ipos, asym):
    pp, fp, rc2, dr2 = o.tables()
    T = o.ptsize + 1
    nt = len(spec["masses"])
    pm = np.zeros((nt, nt), np.int64)
    for k, p in enumerate(spec["pairs"]):
        pm[p[0] - 1, p[1] - 1] = k + 1
        if p[2]:
            pm[p[1] - 1, p[0] - 1] = k + 1
    spring = np.array([p[3] == "spring" for p in spec["pairs"]])
    prm = np.array([list(p[4]) + [0.0] * (4 - len(p[4])) for p in spec["pairs"]])
    pos = np.asarray(spec["pos"], np.float64).reshape(-1, 3)
    box = np.asarray(spec["box"], np.float64)
    typ = np.asarray(spec["typ"], np.int64) - 1
    n = len(pos)
    sr = pos[:, None, :] - pos[None, :, :]
    sr = sr - np.round(sr)
    rij = sr * box
    d2 = rij[..., 0] * rij[..., 0]
    d2 = d2 + rij[..., 1] * rij[..., 1]
    d2 = d2 + rij[..., 2] * rij[..., 2]
    s0 = ipos[:, None, :] - ipos[None, :, :]
    s0 = s0 - np.round(s0)
    r0v = s0 * box
    d20 = r0v[..., 0] * r0v[..., 0]
    d20 = d20 + r0v[..., 1] * r0v[..., 1]
    d20 = d20 + r0v[..., 2] * r0v[..., 2]
    ptij = pm[typ[:, None], typ[None, :]]
    ptji = pm[typ[None, :], typ[:, None]]
    p = np.maximum(ptij, ptji) if asym else ptij
    off = ~np.eye(n, dtype=bool)
    rlist = np.array([prm[k, 0] for k in range(len(prm))]) + spec["control"]["skin"]
    p1 = np.where(p > 0, p - 1, 0)
    inlist = off & (p > 0) & (d2 <= rlist[p1] ** 2)
    isspr = spring[p1]
    # springs
    with np.errstate(divide="ignore", invalid="ignore"):
        r = np.sqrt(d2)
        r0 = np.sqrt(d20)
        sij = r / r0 - 1.0
        fs = prm[p1, 1] * sij * prm[p1, 3] * prm[p1, 3]
        es = 0.5 * fs * sij * r0
        dfs = -fs / r
    sp_ok = inlist & isspr & ~(sij > prm[p1, 2])
    # tables
    tb_ok = inlist & ~isspr & ~(d2 > rc2[p1])
    vdr2 = (1.0 / dr2).astype(np.float32)
    rk = (d2 - 0.25).astype(np.float32) * vdr2[p1] + np.float32(1.0)
    k = np.clip(rk.astype(np.int64), 1, o.ptsize)
    w = rk.astype(np.float64) - k
    base = p1 * T + k - 1
    dft = (w * fp[base + 1] + (1.0 - w) * fp[base]) / np.where(d2 > 0, d2, 1.0)
    et = w * pp[base + 1] + (1.0 - w) * pp[base]
    df = np.where(sp_ok, dfs, np.where(tb_ok, dft, 0.0))
    e = np.where(sp_ok, es, np.where(tb_ok, et, 0.0))
    on_i = (ptji > 0) if asym else np.ones_like(df, bool)
    f = (rij * np.where(on_i, df, 0.0)[..., None]).sum(axis=1)
    count = (ptij == ptji) if asym else np.ones_like(df, bool)
    pe = 0.5 * np.where(count, e, 0.0).sum()
    dv = np.where(count, df, 0.0)
    vir = 0.5 * np.array([(rij[..., a] * rij[..., b] * dv).sum()
                          for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))])
    return f, pe, vir


@pytest.mark.parametrize("onesided", [False, True])
def test_springs_match_all_pairs_rules(onesided):
    spec = W.spring_alloy(5, 300.0, seed=12, quirk="fixed", onesided=onesided)  # 500 atoms
    ipos = np.asarray(spec["pos"], np.float64).reshape(-1, 3).copy()
    spec["pos"] = W.jitter(spec["pos"], spec["box"], 0.08, np.random.default_rng(13))
    o = oracle_from_spec(spec)
    o.init_positions(ipos)
    assert o.setup_lists() == 0
    o.compute(1, 1)  # compute2, or compute3 with the one-sided line
    fo, peo, viro, _ = o.forces()
    fb, peb, virb = _brute(o, spec, ipos, onesided)
    assert rel_l2(fo, fb) < 1e-12
    assert peo == pytest.approx(peb, rel=1e-12)
    assert rel_l2(viro, virb) < 1e-12


def test_unstrained_springs_carry_no_force():
    spec = W.spring_alloy(5, 300.0, seed=14, quirk="fixed", frac2=0.0)  # springs only
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0  # the prologue takes the initial positions
    o.compute(1, 1)
    f, pe, vir, _ = o.forces()
    assert np.abs(f).max() < 1e-12 and abs(pe) < 1e-12

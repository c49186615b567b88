"""The oracle's compute1 (src/nd.f90:364-530), the force routine dynamics
takes when a Pairs line is one-sided ('asym'), pinned on the CPU:

  * with a symmetric PairMat it is compute0 bit for bit (the two differ
    only in how one-sided entries are treated);
  * on a random alloy with a one-sided pair it matches an all-pairs numpy
    evaluation of the same rules (FP32 table index, FP64 tables) within
    1e-12 relative (only the summation order differs).
"""
import numpy as np
import pytest

from helpers import oracle_from_spec, rel_l2
from ndyn_omp_b200 import workloads as W


def test_compute1_equals_compute0_when_symmetric():
    spec = W.cu_crystal(6, 300.0, seed=3, quirk="fixed")
    spec["pos"] = W.jitter(spec["pos"], spec["box"], 0.05, np.random.default_rng(4))
    a = oracle_from_spec(spec)
    a.setup_lists()
    a.compute0(1, 1)
    f0, pe0, v0, _ = a.forces()
    a.L.ora_compute1(a.s, 1, 1)
    f1, pe1, v1, _ = a.forces()
    assert np.array_equal(f0, f1)
    assert pe0 == pe1 and np.array_equal(v0, v1)


def _brute_compute1(o, spec):
    """All pairs i != j, the rules of compute1 applied per ordered pair."""
    pp, fp, rc2, dr2 = o.tables()
    T = o.ptsize + 1
    nt = len(spec["masses"])
    pm = np.zeros((nt, nt), np.int64)  # pm[a-1, b-1] = PairMat(a, b)
    for k, p in enumerate(spec["pairs"]):
        pm[p[0] - 1, p[1] - 1] = k + 1
        if p[2]:
            pm[p[1] - 1, p[0] - 1] = k + 1
    pos = np.asarray(spec["pos"], np.float64).reshape(-1, 3)
    box = np.asarray(spec["box"], np.float64)
    typ = np.asarray(spec["typ"], np.int64) - 1
    n = len(pos)
    sr = pos[:, None, :] - pos[None, :, :]
    sr = sr - np.round(sr)  # anint; no exact halves occur here
    rij = sr * box
    d2 = rij[..., 0] * rij[..., 0]
    d2 = d2 + rij[..., 1] * rij[..., 1]
    d2 = d2 + rij[..., 2] * rij[..., 2]
    ptij = pm[typ[:, None], typ[None, :]]
    ptji = pm[typ[None, :], typ[:, None]]
    mx = np.maximum(ptij, ptji)
    live = (mx > 0) & ~np.eye(n, dtype=bool)
    p1 = np.where(mx > 0, mx - 1, 0)
    live &= ~(d2 > rc2[p1])
    vdr2 = (1.0 / dr2).astype(np.float32)
    rk = (d2 - o_ptrmin(o)).astype(np.float32) * vdr2[p1] + np.float32(1.0)
    k = np.maximum(rk.astype(np.int64), 1)
    w = rk.astype(np.float64) - k
    # live pairs have k <= ptsize; the clip only keeps masked ones in range
    base = p1 * T + np.minimum(k, o.ptsize) - 1
    df = (w * fp[base + 1] + (1.0 - w) * fp[base]) / np.where(d2 > 0, d2, 1.0)
    df = np.where(live, df, 0.0)
    # force on i from j: the pair's i-side applies when PairMat(tj, ti) > 0
    on_i = np.where(ptji > 0, df, 0.0)
    f = (rij * on_i[..., None]).sum(axis=1)
    sym = live & (ptij == ptji)
    e = np.where(sym, w * pp[base + 1] + (1.0 - w) * pp[base], 0.0)
    pe = 0.5 * e.sum()
    dv = np.where(sym, df, 0.0)
    vir = 0.5 * np.array([(rij[..., a] * rij[..., b] * dv).sum()
                          for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))])
    return f, pe, vir


def o_ptrmin(o):
    return 0.25  # the Pairs default, which the workloads use


def test_compute1_matches_all_pairs_rules():
    spec = W.onesided_alloy(6, 300.0, seed=5, quirk="fixed")  # 864 atoms, 3 cells/axis
    spec["pos"] = W.jitter(spec["pos"], spec["box"], 0.05, np.random.default_rng(6))
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0
    o.compute(1, 1)  # dispatches to compute1: one Pairs line is asym
    fo, peo, viro, _ = o.forces()
    fb, peb, virb = _brute_compute1(o, spec)
    assert rel_l2(fo, fb) < 1e-12
    assert peo == pytest.approx(peb, rel=1e-12)
    assert rel_l2(viro, virb) < 1e-12
    # one-sided: the forces no longer cancel
    assert np.linalg.norm(fo.sum(axis=0)) > 1e-6 * np.abs(fo).sum()

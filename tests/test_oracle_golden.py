"""Pin the CPU oracle against the reference's own run logs.

The reference has no unit tests; its known answers are the thermo lines its
example scripts printed (committed under examples/).  tests/golden/
reference_logs.json holds those lines (made by tests/golden/make_golden.py);
here the oracle runs the same scripts on the regenerated lattices and must
print the same numbers to the precision of the log (G14.6 = 6 digits).
"""
import json
import math
import os

import numpy as np
import pytest

import oracle_py
from golden import lattice

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_logs.json")))


def _close(ours, ref, rel, absol):
    return abs(ours - ref) <= max(rel * abs(ref), absol)


def _check_rows(name, rows, ref_rows, ke_rel, press_abs, limit=None):
    assert rows, name
    byref = {r["step"]: r for r in ref_rows}
    n = 0
    for r in rows:
        g = byref.get(r["step"])
        if g is None:
            continue
        n += 1
        # display precision of G14.6 is a half unit in the 6th digit
        assert _close(r["pe"], g["pe"], 6e-6, 0), (name, r, g["text"])
        assert _close(r["vol"], g["vol"], 6e-6, 0), (name, r, g["text"])
        assert _close(r["ke"], g["ke"], ke_rel, 0), (name, r, g["text"])
        assert _close(r["press"], g["press"], 6e-6, press_abs), (name, r, g["text"])
        assert _close(r["eerr"], g["eerr"], 1e-3, 1e-13), (name, r, g["text"])
    assert n >= (limit or 1)


def _run(name, tmp_path, nsteps=None, threads=None):
    case = GOLD[name]
    lattice.materialise(case["model"], str(tmp_path))
    script = list(case["script"])
    if nsteps is not None:
        script = [(" ".join(["Run", str(nsteps)] + ln.split()[2:3]) if ln.split()[:1] == ["Run"]
                   else ln) for ln in script]
    rc, rows, out, err = oracle_py.run_script(script, str(tmp_path), threads=threads)
    assert rc == 0, err
    return rows, case["rows"]


def test_morse_lattice_full_run(tmp_path):
    """examples/MorseTest/out:38-138 -- 4000 steps, every row; the kinetic
    energy here is driven by round-off forces alone and still agrees."""
    rows, ref = _run("MorseTest", tmp_path)
    assert len(rows) == len(ref) == 101
    _check_rows("MorseTest", rows, ref, ke_rel=2e-5, press_abs=0)
    # the printed lines themselves (99 of 101 identical when produced)
    same = sum(a["text"].rstrip() == b["text"].rstrip() for a, b in zip(rows, ref))
    assert same >= 95


def test_soft_potential_lattice(tmp_path):
    """examples/SineTest/out:38 -- the 'soft' table (dpot uses parameters
    1,2 while pot uses 2,3, src/potentials.f90:79,169-170)."""
    rows, ref = _run("SineTest", tmp_path, nsteps=400)
    _check_rows("SineTest", rows, ref, ke_rel=2e-5, press_abs=0, limit=10)


def test_isobaric_relaxation(tmp_path):
    """examples/testT/out:38-57 -- Berendsen barostat (mkIsoP) from the
    Cu lattice: V 49836.0 -> 56637.5, PE -13581.1 -> -12798.8."""
    rows, ref = _run("testT_run1", tmp_path)
    assert len(rows) == 21
    # after convergence the pressure and KE are round-off noise (1e-9)
    _check_rows("testT", rows, ref, ke_rel=5e-3, press_abs=5e-9)
    assert rows[-1]["vol"] == pytest.approx(56637.5, abs=0.06)
    assert rows[-1]["pe"] == pytest.approx(-12798.8, abs=0.06)


@pytest.mark.parametrize("threads,name", [(1, "testCAF_omp1"), (4, "testCAF_omp4")])
def test_large_lattice_skin0(tmp_path, threads, name):
    """examples/testCAF/OMP_4/out_omp1:38 and out_omp4:38: 23328 atoms,
    skin 0 (the list is rebuilt every step); 1 and 4 threads print the
    same line."""
    rows, ref = _run(name, tmp_path, nsteps=3, threads=threads)
    _check_rows(name, rows, ref, ke_rel=2e-3, press_abs=0)
    assert rows[0]["text"].rstrip() == ref[0]["text"].rstrip()


def test_morse_analytic_energy_matches_lammps():
    """examples/MorseTestLmp/log.lammps:54: LAMMPS' analytic Morse energy of
    the same lattice is -13581.418 eV; pot() summed over exact distances
    must give it (the table interpolation then gives -13581.1)."""
    a, n_cells = 3.68, 10
    # distances from one FCC site to all sites within 6.0 A
    rng = np.arange(-3, 4)
    basis = np.array(lattice.BASIS)
    pts = (np.stack(np.meshgrid(rng, rng, rng, indexing="ij"), -1).reshape(-1, 1, 3)
           + basis[None]).reshape(-1, 3) * a
    r = np.linalg.norm(pts, axis=1)
    r = r[(r > 1e-9) & (r <= 6.0)]
    par = [6.0, 0.3429, 1.359, 2.866]
    e_site = sum(oracle_py.pot("morse", x, par) for x in r) / 2.0
    assert 4 * n_cells ** 3 * e_site == pytest.approx(GOLD["MorseTestLmp"]["pe"], abs=5e-4)


def test_table_semantics_at_nodes():
    """buildPairTables (src/potentials.f90:19-33): PPairTable(i) = V(r_i),
    FPairTable(i) = r_i * dpot(r_i) at r_i^2 = PTrMin + (i-1)*dr2."""
    o = oracle_py.Oracle(threads=1)
    o.set_types([63.546, 39.948])
    pairs = [(1, 1, True, "morse", [6.0, 0.3429, 1.3588, 2.866]),
             (2, 2, True, "LJ", [8.5125, 0.0104, 3.405]),
             (1, 2, True, "buck", [8.0, 1500.0, 0.31, 5.0])]
    o.set_pairs(pairs)
    pp, fp, rc2, dr2 = o.tables()
    for j, p in enumerate(pairs):
        assert rc2[j] == p[4][0] ** 2
        assert dr2[j] == (rc2[j] - 0.25) / 999
        for i in (0, 1, 500, 999, 1000):
            s = 0.25 + i * dr2[j]
            r = math.sqrt(s)
            assert pp[1001 * j + i] == oracle_py.pot(p[3], r, p[4])
            assert fp[1001 * j + i] == r * oracle_py.dpot(p[3], r, p[4])
    # analytic closed forms (Morse keeps its extra 1/r, src/potentials.f90:197-198)
    r = 2.9
    D, al, r0 = 0.3429, 1.3588, 2.866
    e = math.exp(-al * (r - r0))
    assert oracle_py.pot("morse", r, pairs[0][4]) == pytest.approx(D * (e * e - 2 * e), rel=1e-14)
    assert oracle_py.dpot("morse", r, pairs[0][4]) == pytest.approx(2 * D * al * (e * e - e) / r,
                                                                     rel=1e-14)
    eps, sig = 0.0104, 3.405
    assert oracle_py.pot("LJ", r, pairs[1][4]) == pytest.approx(
        4 * eps * ((sig / r) ** 12 - (sig / r) ** 6), rel=1e-13)
    assert oracle_py.dpot("buck", r, pairs[2][4]) == pytest.approx(
        1500 * math.exp(-r / 0.31) / 0.31 - 6 * 5 / r ** 7, rel=1e-13)
    assert o.rcut == 8.5125

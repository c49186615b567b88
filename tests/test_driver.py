"""The C++ driver (ndyn_omp_b200/bin/ndyn_gpu) on the reference's own example
scripts: it reads the directive script and model file as read_input does
and must print the reference's logged thermo lines (the committed golden
rows of tests/golden/reference_logs.json) to the precision of the log, as
the CPU oracle does in tests/test_oracle_golden.py.  FP64 path; one
mixed-precision run with the stated force error's effect on energies.
"""
import json
import os
import subprocess

import pytest

from golden import lattice

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "ndyn_omp_b200", "bin", "ndyn_gpu")
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_logs.json")))


def _run(name, tmp_path, nsteps=None, flags=()):
    if not os.path.exists(EXE):
        pytest.fail("driver not built: python -m ndyn_omp_b200.build")
    case = GOLD[name]
    lattice.materialise(case["model"], str(tmp_path))
    script = list(case["script"])
    if nsteps is not None:
        script = [(" ".join(["Run", str(nsteps)] + ln.split()[2:3]) if ln.split()[:1] == ["Run"]
                   else ln) for ln in script]
    r = subprocess.run([EXE, *flags], input="START\n" + "\n".join(script) + "\n", text=True,
                       capture_output=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, r.stderr
    rows = []
    for ln in r.stdout.splitlines():
        w = ln.split()
        if len(w) == 6 and w[0].isdigit():
            rows.append(dict(step=int(w[0]), pe=float(w[1]), ke=float(w[2]), eerr=float(w[3]),
                             press=float(w[4]), vol=float(w[5]), text=ln))
    return rows, case["rows"], r.stdout


def _close(ours, ref, rel, absol):
    return abs(ours - ref) <= max(rel * abs(ref), absol)


def _check(name, rows, ref_rows, ke_rel, press_abs, pe_rel=6e-6, eerr_rel=1e-3, limit=1):
    byref = {r["step"]: r for r in ref_rows}
    n = 0
    for r in rows:
        g = byref.get(r["step"])
        if g is None:
            continue
        n += 1
        assert _close(r["pe"], g["pe"], pe_rel, 0), (name, r, g["text"])
        assert _close(r["vol"], g["vol"], 6e-6, 0), (name, r, g["text"])
        assert _close(r["ke"], g["ke"], ke_rel, 0), (name, r, g["text"])
        assert _close(r["press"], g["press"], 6e-6, press_abs), (name, r, g["text"])
        assert _close(r["eerr"], g["eerr"], eerr_rel, 1e-13), (name, r, g["text"])
    assert n >= limit


def test_driver_morse_lattice(tmp_path):
    """examples/MorseTest/out:38-138: 4000 NVE steps of the Cu lattice."""
    rows, ref, out = _run("MorseTest", tmp_path)
    assert len(rows) == len(ref) == 101
    _check("MorseTest", rows, ref, ke_rel=2e-5, press_abs=0)
    assert "Number of neighbour list updates:       0" in out
    same = sum(a["text"].rstrip() == b["text"].rstrip() for a, b in zip(rows, ref))
    assert same >= 95


def test_driver_isobaric_relaxation(tmp_path):
    """examples/testT/out:38-57: the barostat relaxes V 49836.0 -> 56637.5."""
    rows, ref, _ = _run("testT_run1", tmp_path)
    assert len(rows) == 21
    _check("testT", rows, ref, ke_rel=5e-3, press_abs=5e-9)
    assert rows[-1]["vol"] == pytest.approx(56637.5, abs=0.06)


def test_driver_soft_potential(tmp_path):
    """examples/SineTest/out:38: the 'soft' table."""
    rows, ref, _ = _run("SineTest", tmp_path, nsteps=400)
    _check("SineTest", rows, ref, ke_rel=2e-5, press_abs=0, limit=10)


def test_driver_skin0_large_lattice(tmp_path):
    """examples/testCAF/OMP_4/out_omp1:38: 23328 atoms, skin 0 (a list
    rebuild every step)."""
    rows, ref, _ = _run("testCAF_omp1", tmp_path, nsteps=3)
    _check("testCAF", rows, ref, ke_rel=2e-3, press_abs=0)
    assert rows[0]["text"].rstrip() == ref[0]["text"].rstrip()


def test_driver_mixed_precision(tmp_path):
    """--mixed on the MorseTest lattice: energies within 1e-5 of the log
    (FP32 pair math at <=1e-5 relative force error)."""
    rows, ref, _ = _run("MorseTest", tmp_path, nsteps=400, flags=("--mixed",))
    # the lattice's kinetic energy is round-off noise of the forces, so only
    # the potential energy, pressure and volume are compared
    _check("MorseTest mixed", rows, ref, ke_rel=1e30, press_abs=1e-6, pe_rel=1e-5,
           eerr_rel=1e30, limit=10)


def test_driver_hold_rigid_translation(tmp_path):
    """Hold/Disp through the driver (src/read_input.f90:177-190): holding
    every atom with a displacement on all three axes translates the crystal
    rigidly, so the printed potential energy never changes, while a 'dom rec'
    hold of one slab changes it."""
    case = GOLD["MorseTest"]
    lattice.materialise(case["model"], str(tmp_path))
    base = [ln for ln in case["script"] if ln.split()[:1] not in (["Run"], ["END"])]

    def go(extra):
        script = base + extra + ["OutFreq 20", "Run 100 0.0001", "END"]
        r = subprocess.run([EXE], input="START\n" + "\n".join(script) + "\n", text=True,
                           capture_output=True, cwd=str(tmp_path), timeout=600)
        assert r.returncode == 0, r.stderr
        return [float(ln.split()[1]) for ln in r.stdout.splitlines()
                if len(ln.split()) == 6 and ln.split()[0].isdigit()]

    pe = go(["Hold all typ 1", "Disp all 1.0e-5 -2.0e-5 0.5e-5"])
    assert len(pe) >= 5 and len(set(pe)) == 1
    pe2 = go(["Hold slab dom rec T 0 0 0 0 -0.5 -0.3", "Disp slab 2.0e-4 F F"])
    assert len(set(pe2)) > 1


def test_driver_springs_match_oracle(tmp_path):
    """A 'spring' Pairs line through the driver (compute2 against the
    configuration the first Run starts from, src/nd.f90:104) prints the same
    thermo rows as the oracle's driver on the same script."""
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import oracle_py
    case = GOLD["MorseTest"]
    lattice.materialise(case["model"], str(tmp_path))
    script = ["Model model.dump dump", "NeiMax 200", "Types 1", " Cu 63.546", "Pairs 1",
              " Cu Cu sym spring 3.0 4.0 0.08 1.0", "Seed 99", "Velocity 0.03", "OutFreq 10",
              "Run 60 0.1", "END"]
    r = subprocess.run([EXE], input="START\n" + "\n".join(script) + "\n", text=True,
                       capture_output=True, cwd=str(tmp_path), timeout=600)
    assert r.returncode == 0, r.stderr
    ours = [ln.split() for ln in r.stdout.splitlines()
            if len(ln.split()) == 6 and ln.split()[0].isdigit()]
    rc, ref, _, err = oracle_py.run_script(script, str(tmp_path))
    assert rc == 0, err
    assert len(ours) == len(ref) >= 6
    for a, b in zip(ours, ref):
        assert int(a[0]) == b["step"]
        assert _close(float(a[1]), b["pe"], 2e-6, 1e-9), (a, b["text"])
        assert _close(float(a[2]), b["ke"], 2e-6, 0), (a, b["text"])
    assert float(ours[-1][1]) > 0.0  # the springs are strained by the motion


def _script(name, nsteps, conf):
    case = GOLD[name]
    out = []
    for ln in case["script"]:
        w = ln.split()
        if w[:1] == ["Run"]:
            ln = " ".join(["Run", str(nsteps)] + w[2:3])
        elif w[:1] == ["ConfOutFreq"]:
            ln = conf
        out.append(ln)
    return case, out


def _drive(case, script, where):
    os.makedirs(where, exist_ok=True)
    lattice.materialise(case["model"], where)
    r = subprocess.run([EXE], input="START\n" + "\n".join(script) + "\n", text=True,
                       capture_output=True, cwd=where, timeout=600)
    assert r.returncode == 0, r.stderr
    return [ln for ln in r.stdout.splitlines() if len(ln.split()) == 6 and ln.split()[0].isdigit()]


def test_driver_model_output(tmp_path):
    """write_model every ConfOutFreq steps (src/read_input.f90:394-431,
    src/nd.f90:121,172): the run stops where a model is due and carries on
    (ndg_run_continue), so its thermo lines are the same as one unbroken
    run's.  The dump frames hold the reference's header, the single
    precision positions in f9.5 (xs written as the fractional position,
    the round trip read_model/write_model of the reference), and the xyz
    frames the EN14.4 fields of positions, velocities and a zero energy."""
    import re
    case, one = _script("MorseTest", 200, "ConfOutFreq 0 dump")
    _, five = _script("MorseTest", 200, "ConfOutFreq 50 dump")
    rows_one = _drive(case, one, str(tmp_path / "one"))
    rows_five = _drive(case, five, str(tmp_path / "five"))
    assert rows_one == rows_five and len(rows_one) >= 5
    lines = open(tmp_path / "five" / "out.dump").read().splitlines()
    frames = [k for k, ln in enumerate(lines) if ln == "ITEM: TIMESTEP"]
    assert [int(lines[k + 1]) for k in frames] == [0, 50, 100, 150, 200]
    np_ = int(lines[frames[0] + 3])
    assert np_ == 4000 and lines[frames[0] + 4] == "ITEM: BOX BOUNDS pp pp pp"
    assert lines[frames[0] + 5] == "%12.4f%12.4f" % (0.0, 36.8)
    assert lines[frames[0] + 8] == "ITEM: ATOMS id type xs ys zs"
    model = open(tmp_path / "five" / "model.dump").read().splitlines()
    xs0 = {int(ln.split()[0]): [float(v) for v in ln.split()[2:5]] for ln in model[9:9 + np_]}
    for ln in lines[frames[0] + 9:frames[0] + 9 + np_]:
        assert re.fullmatch(r"[ \d]{7} [ \d]{2}( *-?\d+\.\d{5}){3}", ln), ln
        i, t = int(ln[:7]), int(ln[8:10])
        assert t == 1
        got = [float(ln[10 + 9 * k:19 + 9 * k]) for k in range(3)]
        for a, b in zip(got, xs0[i]):
            assert abs(a - (b - 0.5)) <= 1.5e-5
    _, xyz = _script("MorseTest", 100, "ConfOutFreq 50 xyz")
    _drive(case, xyz, str(tmp_path / "xyz"))
    lines = open(tmp_path / "xyz" / "out.xyz").read().splitlines()
    assert len(lines) == 3 * (2 + 4000) and int(lines[0]) == 4000 and lines[1] == ""
    en = re.compile(r" *-?\d{1,3}\.\d{4}E[+-]\d{2}")
    for ln in lines[2:4002] + lines[-4000:]:
        assert ln[:5] == "Cu   " and len(ln) == 5 + 7 * 14, ln
        fields = [ln[5 + 14 * k:19 + 14 * k] for k in range(7)]
        for f in fields:
            assert en.fullmatch(f), ln
            m = float(f.strip().split("E")[0])
            assert m == 0.0 or 1.0 <= abs(m) < 1000.0, f
        assert fields[6].strip() == "0.0000E+00"
        assert all(abs(float(f)) <= 0.5001 for f in fields[:3])

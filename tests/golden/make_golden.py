"""Generate tests/golden/reference_logs.json from the reference's own run logs.

The reference (stewmasterj/Ndyn_OMP) has no unit tests; its known answers are
the committed outputs of its example scripts.  This script reads those logs
from a checkout of the reference and stores, for each pinned example:

  * the directive script (the lines between START and END, as run),
  * the model the script reads, described by the lattice that regenerates it
    (the dump files are perfect FCC lattices, so they are rebuilt in the
    tests instead of being copied),
  * every thermo row the log printed (step, PE, KE, energy error, pressure,
    volume), and the source file:line of each row.

Usage:  python tests/golden/make_golden.py /path/to/reference
The output is committed; the tests never read the reference at run time.
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

CASES = {
    # examples/MorseTest: Cu FCC a=3.68, 4000 atoms, Morse, default skin
    "MorseTest": {
        "script": "examples/MorseTest/input.sh",
        "log": "examples/MorseTest/out",
        "model": {"kind": "fcc_dump", "cells": 10, "box": 36.8, "file": "model.dump"},
    },
    # examples/testT run 1: the deterministic isobaric relaxation
    "testT_run1": {
        "script": "examples/testT/input.sh",
        "log": "examples/testT/out",
        "model": {"kind": "fcc_dump", "cells": 10, "box": 36.8,
                  "file": "../MorseTest/model.dump"},
        "first_run_only": True,
    },
    # examples/SineTest: 'soft' potential on the same lattice
    "SineTest": {
        "script": "examples/SineTest/input.sh",
        "log": "examples/SineTest/out",
        "model": {"kind": "fcc_dump", "cells": 10, "box": 36.8, "file": "model.dump"},
    },
    # examples/testCAF/OMP_4: 18^3 FCC Cu a=3.629 (box 65.322), skin 0,
    # one thread and four threads give the same line
    "testCAF_omp1": {
        "script": "examples/testCAF/OMP_4/input.sh",
        "log": "examples/testCAF/OMP_4/out_omp1",
        "model": {"kind": "fcc_xyz", "cells": 18, "a": 3.629, "lo": -9,
                  "type": "Cu", "file": "../model.xyz"},
    },
    "testCAF_omp4": {
        "script": "examples/testCAF/OMP_4/input.sh",
        "log": "examples/testCAF/OMP_4/out_omp4",
        "model": {"kind": "fcc_xyz", "cells": 18, "a": 3.629, "lo": -9,
                  "type": "Cu", "file": "../model.xyz"},
    },
}

ROW = re.compile(r"^\s+(\d+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s*$")


def fnum(s):
    return float(s.replace("D", "E"))


def read_script(path):
    lines, on = [], False
    for ln in open(path):
        w = ln.split()
        if not on:
            if w and w[0] == "START":
                on = True
            continue
        lines.append(ln.rstrip("\n"))
        if w and w[0] in ("END", "DONE", "end", "done"):
            break
    return lines


def read_rows(path, first_run_only):
    rows, runs = [], 0
    for no, ln in enumerate(open(path), 1):
        if ln.startswith("#  Step"):
            runs += 1
            if first_run_only and runs > 1:
                break
            continue
        m = ROW.match(ln)
        if m and runs:
            step, pe, ke, ee, p, v = m.groups()
            rows.append({"step": int(step), "pe": fnum(pe), "ke": fnum(ke),
                         "eerr": fnum(ee), "press": fnum(p), "vol": fnum(v),
                         "text": ln.rstrip("\n"), "src": f"{path_rel(path)}:{no}"})
    return rows


def path_rel(p):
    return p.split("/examples/", 1)[-1] if "/examples/" in p else p


def main(ref):
    out = {"_about": "Known-answer rows from the reference's committed example logs; "
                     "generated by tests/golden/make_golden.py"}
    for name, c in CASES.items():
        script = read_script(os.path.join(ref, c["script"]))
        if c.get("first_run_only"):
            cut = []
            for ln in script:
                cut.append(ln)
                if ln.split()[:1] == ["Run"]:
                    break
            script = cut + ["END"]
        out[name] = {
            "script_src": c["script"],
            "script": script,
            "model": c["model"],
            "rows": read_rows(os.path.join(ref, c["log"]), c.get("first_run_only", False)),
        }
    # LAMMPS analytic cross-check on the MorseTest lattice (no table)
    for no, ln in enumerate(open(os.path.join(ref, "examples/MorseTestLmp/log.lammps")), 1):
        w = ln.split()
        if len(w) == 6 and w[0] == "0" and w[1] == "0":
            out["MorseTestLmp"] = {"pe": float(w[2]), "press_bar": float(w[5]),
                                   "src": f"MorseTestLmp/log.lammps:{no}"}
            break
    with open(os.path.join(HERE, "reference_logs.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "reference_logs.json"))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])

"""A device allocation that fails (host-side fault injection: the library's
NDG_TEST_ALLOC_LIMIT hook fails every device allocation above a size, as a
full device would; no GPU fault is involved).

A context whose list arena cannot grow for a newly added system reports
NDG_ERR_NOMEM from the list build that needs it (not a CUDA error on some
later call) and stays consistent: after the new system is removed, its other
system runs on to the same bits as in a context that took the same steps
without the failed build.
Each case runs in a child process: the hook is read once per process.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
import ndyn_omp_b200 as nd
from ndyn_omp_b200 import workloads as W
from helpers import gpu_from_spec
out = {}
with nd.Context(0, "mixed") as ctx:
    a = gpu_from_spec(ctx, W.ar_liquid(6, 120.0, seed=81, quirk="fixed"))     # 864 atoms
    ctx.run(20)
    b = gpu_from_spec(ctx, W.ar_liquid(10, 120.0, seed=82, quirk="fixed"))    # 4000 atoms
    out["status"] = 0
    if sys.argv[3] == "try":
        try:
            ctx.setup_lists()  # the prologue for the new system: the list arena grows
        except nd.NdgError as e:
            out["status"] = e.status
    # both children go on alike: the new system leaves, lists are built again
    ctx.remove_system(b)
    ctx.setup_lists()
    ctx.run(20, cont=True)
    ctx.run(20, cont=True)
    pos, vel, acc, box = ctx.state(a)
np.savez(sys.argv[2], pos=pos, vel=vel, acc=acc, box=box)
print(json.dumps(out))
'''


def _child(tmp_path, limit):
    env = dict(os.environ)
    env.pop("NDG_TEST_ALLOC_LIMIT", None)
    if limit:
        env["NDG_TEST_ALLOC_LIMIT"] = str(limit)
    npz = os.path.join(str(tmp_path), f"state_{limit}.npz")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, npz, "try" if limit else "skip"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1]), np.load(npz)


def test_list_arena_growth_failure_is_nomem_and_context_survives(tmp_path):
    NDG_ERR_NOMEM = -6
    ok, s_ok = _child(tmp_path, 0)
    # 1 MB: the 864-atom system's arrays fit (its list block ~0.4 MB), the
    # list arena for the 4000-atom one (~2 MB) does not
    bad, s_bad = _child(tmp_path, 1 << 20)
    assert bad["status"] == NDG_ERR_NOMEM
    # the surviving system took the same steps and list builds in both
    for k in ("pos", "vel", "acc", "box"):
        assert np.array_equal(s_ok[k], s_bad[k]), k

"""Hold groups with displacement conditions in the oracle's integrate1
(src/nd.f90:1048-1077): a held atom's constrained components move by the
group's displacement per step, every other component (and every other
atom) by its velocity, exactly as the Nhold == 0 branch moves it."""
import numpy as np

from helpers import oracle_from_spec
from ndyn_omp_b200 import workloads as W


def test_integrate1_hold_branch():
    spec = W.onesided_alloy(6, 600.0, seed=9, quirk="fixed")
    rng = np.random.default_rng(10)
    spec["acc"] = rng.standard_normal(spec["pos"].shape) * 1e-3
    n = len(spec["typ"])
    hold = np.zeros(n, np.int32)
    hold[: n // 3] = 1
    hold[n // 3: n // 2] = 2          # a group with no constrained axis
    dirs = [[True, False, True], [False, False, False]]
    du = [[1.5e-4, 0.0, -2.0e-4], [0.0, 0.0, 0.0]]

    free = oracle_from_spec(spec)
    free.setup_lists()
    free.integrate1()
    pf, _, _, _ = free.state()

    held = oracle_from_spec(spec)
    held.set_holds(hold, dirs, du)
    held.setup_lists()
    held.integrate1()
    ph, _, _, _ = held.state()

    p0 = np.asarray(spec["pos"], np.float64).reshape(-1, 3)
    g1 = hold == 1
    assert np.array_equal(ph[g1, 0], p0[g1, 0] + 1.5e-4)
    assert np.array_equal(ph[g1, 2], p0[g1, 2] + (-2.0e-4))
    assert np.array_equal(ph[g1, 1], pf[g1, 1])
    assert np.array_equal(ph[~g1], pf[~g1])

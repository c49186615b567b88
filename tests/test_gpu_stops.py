"""The reference's STOPs as status codes, from host-made inputs (no GPU fault
is involved: every write the failing kernels make is bounded).

  * 'too many neighbours in list' (buildVerletList, src/nd.f90:1378,1421):
    in the reference semantics an atom's half list may not exceed NeiMax,
    the caller's or the reference's estimate (src/nd.f90:84-88).  The GPU
    stops at exactly the NeiMax values the oracle stops at, on grids of
    three cells and of two (where the half stencil visits a cell twice).
    In either semantics a list longer than the device capacity (atoms packed
    far above the mean density) stops as well.
  * 'Particle outside of box' (CheckListUpdate, src/nd.f90:1494): two
    fractional displacements whose squared sum exceeds one box.
"""
import numpy as np
import pytest

from helpers import gpu_from_spec, oracle_from_spec

pytestmark = pytest.mark.gpu

nd = pytest.importorskip("ndyn_omp_b200")
from ndyn_omp_b200 import workloads as W  # noqa: E402

NDG_ERR_NEIMAX, NDG_ERR_OUT_OF_BOX = -2, -3


def _spec(name):
    rng = np.random.default_rng(71)
    if name == "cu3":     # 864 atoms, 3 cells per axis
        sp = W.cu_crystal(6, 300.0, seed=72, quirk="ref")
    elif name == "cu2":   # 500 atoms, 2 cells per axis: the stencil repeats cells
        sp = W.cu_crystal(5, 300.0, seed=73, quirk="ref")
    else:                 # two types, three pair potentials
        sp = W.nacl_solid((4, 4, 4), 300.0, seed=74, quirk="ref")
    sp["pos"] = W.jitter(sp["pos"], sp["box"], 0.1, rng)
    return sp


def _oracle_rc(spec, neimax):
    sp = dict(spec, control=dict(spec["control"], neimax=neimax))
    return oracle_from_spec(sp).setup_lists()


def _gpu_rc(spec, neimax, nsteps=0):
    sp = dict(spec, control=dict(spec["control"], neimax=neimax))
    with nd.Context(0, "fp64") as ctx:
        gpu_from_spec(ctx, sp)
        try:
            if nsteps:
                ctx.run(nsteps)
            else:
                ctx.setup_lists()
        except nd.NdgError as e:
            return e.status
    return 0


@pytest.mark.parametrize("name", ["cu3", "cu2", "nacl"])
def test_neimax_stop_matches_oracle(name):
    spec = _spec(name)
    # the smallest NeiMax the oracle builds the lists with
    lo, hi = 1, 2000
    assert _oracle_rc(spec, hi) == 0
    while lo < hi:
        mid = (lo + hi) // 2
        if _oracle_rc(spec, mid) == 0:
            hi = mid
        else:
            lo = mid + 1
    h = lo
    assert _oracle_rc(spec, h - 1) == NDG_ERR_NEIMAX
    assert _gpu_rc(spec, h) == 0
    assert _gpu_rc(spec, h - 1) == NDG_ERR_NEIMAX
    # the run stops as well (its prologue builds the lists)
    assert _gpu_rc(spec, h - 1, nsteps=5) == NDG_ERR_NEIMAX
    assert _gpu_rc(spec, h, nsteps=5) == 0


def test_neimax_estimate_default():
    """NeiMax 0: the reference's estimate applies (and is kept, as the
    module variable keeps it)."""
    spec = _spec("cu3")
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0
    with nd.Context(0, "fp64") as ctx:
        sid = gpu_from_spec(ctx, spec)
        ctx.setup_lists()
        assert ctx.control(sid).neimax == o.neimax > 0


@pytest.mark.parametrize("quirk", ["ref", "fixed"])
def test_capacity_stop_on_packed_atoms(quirk):
    """Every atom packed into one octant of the box (eight times the mean
    density): the lists outgrow both the reference's NeiMax estimate and
    the device capacity sized from the mean density."""
    spec = W.cu_crystal(8, 300.0, seed=75, quirk=quirk)
    spec["pos"] = (np.asarray(spec["pos"]) + 0.5) * 0.5 - 0.5
    assert oracle_from_spec(spec).setup_lists() == NDG_ERR_NEIMAX
    for prec in ("fp64", "mixed"):
        with nd.Context(0, prec) as ctx:
            gpu_from_spec(ctx, spec)
            with pytest.raises(nd.NdgError) as e:
                ctx.setup_lists()
            assert e.value.status == NDG_ERR_NEIMAX


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_particle_outside_of_box(prec):
    """One atom moving more than a box length in one step: the reference
    semantics' CheckListUpdate stops the run."""
    spec = W.cu_crystal(6, 300.0, seed=76, quirk="ref")
    vel = np.array(spec["vel"], np.float64)
    vel[0] = [400.0, 0.0, 0.0]  # 40 A per step in a 21.7 A box
    spec["vel"] = vel
    o = oracle_from_spec(spec)
    rc, _ = o.run(5, spec["control"]["dt"])
    assert rc == NDG_ERR_OUT_OF_BOX
    with nd.Context(0, prec) as ctx:
        gpu_from_spec(ctx, spec)
        with pytest.raises(nd.NdgError) as e:
            ctx.run(5)
        assert e.value.status == NDG_ERR_OUT_OF_BOX

"""ndg_compute0_static: compute0 for callers that cannot allocate device memory.

Such callers are host applications whose own memory pool owns the GPU and
only lends out buffers, and loops that must not stall on cudaMalloc/cudaFree.
They hand in device buffers they already hold; the entry point keeps its
scratch in a static device array.  Here torch plays that caller: it owns the
input and output buffers.  On two consecutive calls the result must equal
the context path (ndg_compute) and the CPU oracle's compute0 (compute1 for a
one-sided pair) within the FP64 tolerance of the other parity tests, and the
device's free memory must not move across a call.  The file is collected
last.
"""
import ctypes

import numpy as np
import pytest

from helpers import oracle_from_spec

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12  # the FP64 force tolerance of tests/test_gpu_parity.py


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _cases():
    from ndyn_omp_b200 import workloads as W
    rng = np.random.default_rng(44)
    cu = W.cu_crystal(8, 300.0, seed=41, quirk="ref")
    cu["pos"] = W.jitter(cu["pos"], cu["box"], 0.05, rng)
    alloy = W.onesided_alloy(8, 300.0, seed=46, quirk="fixed")
    alloy["pos"] = W.jitter(alloy["pos"], alloy["box"], 0.05, rng)
    return [cu,                                                  # 2048 atoms, one pair
            W.nacl_solid((6, 6, 6), 600.0, seed=42, quirk="fixed"),  # two types, three pairs
            W.cu_crystal(5, 900.0, seed=43, quirk="ref"),           # 2 link cells: repeats
            W.ar_liquid(14, 120.0, seed=45, quirk="fixed"),         # 10976 atoms
            alloy]                                               # one-sided (asym) pair


def _static_inputs(spec):
    import torch

    import ndyn_omp_b200 as nd
    n = len(spec["typ"])
    ntypes, npairs = len(spec["masses"]), len(spec["pairs"])
    pp, fp, _, _ = nd.build_pair_tables(spec["pairs"])
    pm = nd.pair_matrix(spec["pairs"], ntypes).astype(np.int32)
    rcp = np.array([p[4][0] for p in spec["pairs"]], np.float64)
    box = np.ascontiguousarray(spec["box"], np.float64)
    dev = torch.device("cuda", 0)
    return dict(
        n=n, ntypes=ntypes, npairs=npairs, pm=pm, rcp=rcp, box=box,
        pos_d=torch.tensor(np.ascontiguousarray(spec["pos"]).ravel(), dtype=torch.float64,
                           device=dev),
        typ_d=torch.tensor(np.asarray(spec["typ"], np.int32), device=dev),
        fp_d=torch.tensor(fp, dtype=torch.float64, device=dev),
        pp_d=torch.tensor(pp, dtype=torch.float64, device=dev),
        force_d=torch.empty(3 * n, dtype=torch.float64, device=dev))


def _call(L, a, skin, quirk, stream, typ_d=None):
    pe = ctypes.c_double(float("nan"))
    vir = np.full(6, np.nan)
    rc = L.ndg_compute0_static(a["n"], a["ntypes"], a["npairs"], 1000, 0.25, _p(a["pm"]),
                               _p(a["rcp"]), float(skin), quirk, _p(a["box"]),
                               a["fp_d"].data_ptr(), a["pp_d"].data_ptr(),
                               a["pos_d"].data_ptr(),
                               (a["typ_d"] if typ_d is None else typ_d).data_ptr(),
                               a["force_d"].data_ptr(), ctypes.byref(pe), _p(vir), stream)
    return rc, pe.value, vir


@pytest.mark.parametrize("case", range(5))
def test_static_compute0_matches_context_and_oracle(case):
    import torch

    import ndyn_omp_b200 as nd
    L = nd.lib()
    spec = _cases()[case]
    ctl = spec["control"]
    quirk = 0 if ctl.get("quirk", "ref") == "ref" else 1
    # the existing entry point: a context, its lists, compute0
    with nd.Context(0, "fp64") as ctx:
        sid = ctx.add_system(spec["masses"], spec["pairs"], spec["typ"], spec["pos"],
                             spec["box"], vel=spec.get("vel"))
        ctx.set_control(sid, **ctl)
        ctx.setup_lists()
        skin = ctx.control(sid).skin
        ctx.compute0(True, True)
        f_ref, pe_ref, vir_ref, _ = ctx.forces(sid)
    # the oracle: compute0, or compute1 where a pair is one-sided
    o = oracle_from_spec(spec)
    assert o.setup_lists() == 0
    assert abs(o.skin - skin) <= 1e-15 * skin
    o.compute(1, 1)
    f_o, pe_o, vir_o, _ = o.forces()
    # the allocation-free entry point on caller-owned device buffers
    a = _static_inputs(spec)
    n = a["n"]
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        a["force_d"].fill_(float("nan"))
        torch.cuda.synchronize(dev)
        free0, _ = torch.cuda.mem_get_info(dev)
        rc, pe, vir = _call(L, a, skin, quirk, stream)
        free1, _ = torch.cuda.mem_get_info(dev)
        assert rc == 0, (call, rc)
        if call == 1:
            # the first call on a device may load the library's device code,
            # which brings the static array with it; later calls take nothing
            assert free1 == free0, (call, free0 - free1)
        f = a["force_d"].cpu().numpy().reshape(n, 3)
        for f_cmp, pe_cmp, vir_cmp in ((f_ref, pe_ref, vir_ref), (f_o, pe_o, vir_o)):
            assert _rel(f, f_cmp) < FP64_TOL, call
            assert abs(pe - pe_cmp) <= FP64_TOL * abs(pe_cmp), call
            assert _rel(vir, vir_cmp) < FP64_TOL, call


def test_static_compute0_rejects_bad_inputs():
    import torch

    import ndyn_omp_b200 as nd
    L = nd.lib()
    dev = torch.device("cuda", 0)
    spec = _cases()[0]
    a = _static_inputs(spec)
    stream = torch.cuda.current_stream(dev).cuda_stream
    # an atom type outside 1..ntypes: flagged on the device, left out of the
    # sums, and the call says so
    bad = a["typ_d"].clone()
    bad[17] = 0
    rc, _, _ = _call(L, a, 0.5, 0, stream, typ_d=bad)
    assert rc == -1  # NDG_ERR_ARG
    bad[17] = 5
    rc, _, _ = _call(L, a, 0.5, 0, stream, typ_d=bad)
    assert rc == -1
    # a good call right after leaves no trace of the flag
    rc, _, _ = _call(L, a, 0.5, 0, stream)
    assert rc == 0
    # negative skin, and a box whose cell count would not fit an int: refused
    # on the host before any device work
    rc, _, _ = _call(L, a, -0.5, 0, stream)
    assert rc == -1
    big = dict(a, box=np.array([1e12, 1e12, 1e12]))
    rc, _, _ = _call(L, big, 0.5, 0, stream)
    assert rc == -1
    # a box under two cells per axis: the reference's minimum image fails
    small = dict(a, box=np.array([10.0, 10.0, 10.0]))
    rc, _, _ = _call(L, small, 0.5, 0, stream)
    assert rc == -5  # NDG_ERR_CELLS


def test_static_compute0_rejects_oversize():
    import torch

    import ndyn_omp_b200 as nd
    L = nd.lib()
    n = 40000  # above the 32768-atom limit: refused before any device work
    pm = np.ones(1, np.int32)
    rcp = np.array([6.0])
    box = np.array([100.0, 100.0, 100.0])
    pe = ctypes.c_double()
    vir = np.zeros(6)
    dev = torch.device("cuda", 0)
    tab = torch.zeros(1001, dtype=torch.float64, device=dev)
    pos_d = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    typ_d = torch.ones(n, dtype=torch.int32, device=dev)
    force_d = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    rc = L.ndg_compute0_static(n, 1, 1, 1000, 0.25, _p(pm), _p(rcp), 0.5, 0, _p(box),
                               tab.data_ptr(), tab.data_ptr(), pos_d.data_ptr(),
                               typ_d.data_ptr(), force_d.data_ptr(), ctypes.byref(pe), _p(vir),
                               None)
    assert rc == -1  # NDG_ERR_ARG

"""ndg_compute0_static: compute0 for callers that cannot allocate device memory.

Such callers (code issuing work during CUDA stream capture, applications
that own all device memory through their own pool, latency-bound loops)
hand in device buffers they already hold; the entry point keeps its scratch
in a static device array.  Here torch plays that caller: it owns the input
and output buffers, and the result must equal the context path
(ndg_compute) within the FP64 tolerance of the other parity tests, on two
consecutive calls.  The file is collected last.
"""
import ctypes

import numpy as np
import pytest

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
    return [cu,                                                  # 2048 atoms, one pair
            W.nacl_solid((6, 6, 6), 600.0, seed=42, quirk="fixed"),  # two types, three pairs
            W.cu_crystal(5, 900.0, seed=43, quirk="ref"),           # 2 link cells: repeats
            W.ar_liquid(14, 120.0, seed=45, quirk="fixed")]         # 10976 atoms


@pytest.mark.parametrize("case", range(4))
def test_static_compute0_matches_context(case):
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
    # the allocation-free entry point on caller-owned device buffers
    n = len(spec["typ"])
    ntypes, npairs = len(spec["masses"]), len(spec["pairs"])
    pp, fp, _, _ = nd.build_pair_tables(spec["pairs"])
    pm = nd.pair_matrix(spec["pairs"], ntypes).astype(np.int32)
    rcp = np.array([p[4][0] for p in spec["pairs"]], np.float64)
    box = np.ascontiguousarray(spec["box"], np.float64)
    dev = torch.device("cuda", 0)
    pos_d = torch.tensor(np.ascontiguousarray(spec["pos"]).ravel(), dtype=torch.float64,
                         device=dev)
    typ_d = torch.tensor(np.asarray(spec["typ"], np.int32), device=dev)
    fp_d = torch.tensor(fp, dtype=torch.float64, device=dev)
    pp_d = torch.tensor(pp, dtype=torch.float64, device=dev)
    force_d = torch.empty(3 * n, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        force_d.fill_(float("nan"))
        pe = ctypes.c_double(float("nan"))
        vir = np.full(6, np.nan)
        rc = L.ndg_compute0_static(n, ntypes, npairs, 1000, 0.25, _p(pm), _p(rcp), float(skin),
                                   quirk, _p(box), fp_d.data_ptr(), pp_d.data_ptr(),
                                   pos_d.data_ptr(), typ_d.data_ptr(), force_d.data_ptr(),
                                   ctypes.byref(pe), _p(vir), stream)
        assert rc == 0, (call, rc)
        f = force_d.cpu().numpy().reshape(n, 3)
        assert _rel(f, f_ref) < FP64_TOL, call
        assert abs(pe.value - pe_ref) <= FP64_TOL * abs(pe_ref), call
        assert _rel(vir, vir_ref) < FP64_TOL, call


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

"""CPU-side checks of the C ABI library: it loads, exports every symbol
include/ndyn_gpu.h declares, and its host-side table builder reproduces the
oracle's buildPairTables bit for bit.  No GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_py

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ndyn_gpu.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ndg_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from ndyn_omp_b200 import _lib
    return _lib.lib()


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_abi_version_and_errors(lib):
    assert lib.ndg_abi_version() == 1
    assert lib.ndg_error_string(-2) == b"too many neighbours in list"
    assert lib.ndg_error_string(-3) == b"Particle outside of box"


def test_create_without_gpu_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    c = ctypes.c_void_p()
    assert lib.ndg_create(ctypes.byref(c), 0, 0) == -7  # NDG_ERR_CUDA, no CPU fallback


PAIRS = [(1, 1, True, "morse", [6.0, 0.3429, 1.3588, 2.866]),
         (2, 2, True, "LJ", [8.5125, 0.0104, 3.405]),
         (1, 2, True, "buck", [8.0, 1500.0, 0.31, 5.0]),
         (1, 1, True, "soft", [6.0, 0.5, 6.0]),
         (1, 1, True, "MorseC", [6.0, 0.3429, 1.359, 2.866]),
         (1, 1, True, "John", [5.0, 0.2, 2.5, 5.0])]


@pytest.mark.parametrize("ptsize,ptrmin", [(1000, 0.25), (2000, 0.5), (333, 0.1)])
def test_tables_bit_exact_vs_oracle(ptsize, ptrmin):
    from ndyn_omp_b200 import build_pair_tables
    charges = [0.5, -0.5]
    pp, fp, rc2, dr2 = build_pair_tables(PAIRS, ptsize, ptrmin, charges=charges)
    o = oracle_py.Oracle(threads=1)
    o.set_types([63.5, 40.0])
    o.set_pairs(PAIRS, ptrmin, ptsize, charges=charges)
    opp, ofp, orc2, odr2 = o.tables()
    assert np.array_equal(pp, opp)
    assert np.array_equal(fp, ofp)
    assert np.array_equal(rc2, orc2)
    assert np.array_equal(dr2, odr2)


def test_unknown_potential_rejected():
    from ndyn_omp_b200 import NdgError, build_pair_tables
    with pytest.raises(NdgError) as e:
        build_pair_tables([(1, 1, True, "mors", [6.0, 1, 1, 1])])
    assert e.value.status == -4


def test_pair_matrix_layout():
    from ndyn_omp_b200 import pair_matrix
    pm = pair_matrix([(1, 1, True, "a", [1]), (2, 2, True, "b", [1]), (1, 2, True, "c", [1])], 2)
    # column-major PairMat(a,b) at (a-1)+(b-1)*ntypes
    assert list(pm) == [1, 3, 3, 2]


def test_bench_script_compiles():
    """bench.py (run by the driver on the GPU host) is valid Python"""
    import ast
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ast.parse(open(os.path.join(root, "bench.py")).read())

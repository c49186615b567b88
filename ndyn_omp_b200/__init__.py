"""B200-native (sm_100a) implementation of Ndyn's MD timestep path.

The compute path is the CUDA library ndyn_omp_b200/lib/libndyn_gpu.so
(C ABI: include/ndyn_gpu.h); this package is its Python host mirror.
"""
from ._lib import LIB_PATH, lib  # noqa: F401
from .api import (Context, Control, NdgError, Server, Thermo, admit_plan,  # noqa: F401
                  build_pair_tables, make_control, pair_matrix)

__all__ = ["Context", "Control", "NdgError", "Server", "Thermo", "admit_plan",
           "build_pair_tables", "make_control", "pair_matrix", "lib", "LIB_PATH"]

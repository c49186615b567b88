"""Loader of the in-tree CUDA library (ndyn_omp_b200/lib/libndyn_gpu.so).

There is no fallback: if the library is missing or cannot be loaded, every
call raises.  build() compiles it with nvcc for sm_100a.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libndyn_gpu.so")
_lib = None

# the C ABI of include/ndyn_gpu.h: (name, restype, argtypes)
vp, i, d, ll = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_longlong
SIGNATURES = [
    ("ndg_abi_version", i, []),
    ("ndg_error_string", ctypes.c_char_p, [i]),
    ("ndg_last_error", ctypes.c_char_p, [vp]),
    ("ndg_build_pair_tables", i, [i, i, d, ctypes.c_char_p, vp, vp, vp, vp, vp, vp]),
    ("ndg_create", i, [vp, i, i]),
    ("ndg_destroy", i, [vp]),
    ("ndg_set_precision", i, [vp, i]),
    ("ndg_add_system", i, [vp, i, i, i, i, d, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]),
    ("ndg_remove_system", i, [vp, i]),
    ("ndg_num_systems", i, [vp]),
    ("ndg_load_state", i, [vp, i, vp, vp, vp, vp]),
    ("ndg_get_state", i, [vp, i, vp, vp, vp, vp]),
    ("ndg_set_control", i, [vp, i, vp]),
    ("ndg_set_holds", i, [vp, i, vp, i, vp, vp]),
    ("ndg_set_springs", i, [vp, i, vp, vp]),
    ("ndg_set_initial_positions", i, [vp, i, vp, vp]),
    ("ndg_get_control", i, [vp, i, vp]),
    ("ndg_default_control", None, [vp]),
    ("ndg_setup_lists", i, [vp]),
    ("ndg_build_cell_list", i, [vp]),
    ("ndg_check_list_update", i, [vp, vp]),
    ("ndg_integrate1", i, [vp]),
    ("ndg_compute", i, [vp, i, i]),
    ("ndg_integrate2", i, [vp, i]),
    ("ndg_mk_iso_ke", i, [vp, i]),
    ("ndg_mk_iso_e", i, [vp, i]),
    ("ndg_mk_iso_p", i, [vp, i]),
    ("ndg_get_forces", i, [vp, i, vp, vp, vp, vp]),
    ("ndg_run", i, [vp, i, vp, vp]),
    ("ndg_run_continue", i, [vp, i, vp, vp]),
    ("ndg_get_thermo", i, [vp, i, vp]),
    ("ndg_get_list_updates", i, [vp, i, vp]),
    ("ndg_get_mcell", i, [vp, i, vp]),
    ("ndg_get_cells", i, [vp, i, vp]),
    ("ndg_get_neighbors", i, [vp, i, vp, ll, vp]),
    ("ndg_get_neighbor_count", i, [vp, i, vp]),
    ("ndg_set_tuning", i, [vp, i, i]),
    ("ndg_get_tuning", i, [vp, vp, vp]),
    ("ndg_set_gather_depth", i, [vp, i]),
    ("ndg_get_gather_depth", i, [vp, vp]),
    ("ndg_set_list_split", i, [vp, i, i]),
    ("ndg_get_list_split", i, [vp, vp, vp]),
    ("ndg_autotune", i, [vp, i]),
    ("ndg_autotune_skin", i, [vp, i, vp]),
    ("ndg_device_bytes", i, [vp, vp]),
    ("ndg_system_bytes", ll, [i, i, i, i, d, d, i]),
    ("ndg_get_kernel_times", i, [vp, vp, vp, vp, vp]),
    ("ndg_get_stream", i, [vp, vp]),
    ("ndg_profile_run", i, [vp, i]),
    ("ndg_server_create", i, [vp, i, i, ll, i]),
    ("ndg_server_destroy", i, [vp]),
    ("ndg_server_submit", i, [vp, vp, vp]),
    ("ndg_server_step", i, [vp, vp]),
    ("ndg_server_poll", i, [vp, vp, i, vp]),
    ("ndg_server_status", i, [vp, ll, vp]),
    ("ndg_server_result", i, [vp, ll, vp, vp, vp, vp, vp, i, vp]),
    ("ndg_server_stats_get", i, [vp, vp]),
    ("ndg_server_context", i, [vp, vp]),
    ("ndg_admit_plan", i, [vp, i, ll, ll, vp]),
    ("ndg_compute0_static", i, [i, i, i, i, d, vp, vp, d, i, vp, vp, vp, vp, vp, vp, vp, vp,
                                vp]),
]


def lib():
    """Load the library once; raise if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"CUDA library not built: {LIB_PATH} (run python -m "
                               "ndyn_omp_b200.build)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib

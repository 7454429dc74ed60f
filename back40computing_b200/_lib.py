"""ctypes binding of libb40c_bfs.so (declarations in include/b40c_bfs.h).

The library is the product: every search runs its sm_100a kernels.  There is no
fallback -- importing this module fails loudly when the shared object has not
been built (``python -m back40computing_b200.build``).
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int64, c_longlong, c_uint64, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libb40c_bfs.so"


class CsrT(ctypes.Structure):
    """struct b40c_csr (include/b40c_bfs.h)."""
    _fields_ = [("nodes", c_int64), ("edges", c_int64),
                ("row_offsets", POINTER(c_int)), ("column_indices", POINTER(c_int))]


# name -> (restype, argtypes).  Every symbol the header declares.
SIGNATURES = {
    "b40c_last_error_string": (c_char_p, []),
    "b40c_version": (c_char_p, []),
    "b40c_problem_create": (c_int, [c_int, POINTER(c_void_p)]),
    "b40c_problem_destroy": (c_int, [c_void_p]),
    "b40c_problem_from_host": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int]),
    "b40c_problem_reset": (c_int, [c_void_p, c_int, c_double]),
    "b40c_problem_reset_async": (c_int, [c_void_p, c_int, c_double]),
    "b40c_problem_extract_results": (c_int, [c_void_p, c_void_p]),
    "b40c_problem_extract_results_async": (c_int, [c_void_p, c_void_p]),
    "b40c_problem_set_label_buffers": (c_int, [c_void_p, c_int]),
    "b40c_problem_sync": (c_int, [c_void_p]),
    "b40c_problem_from_host_ids64": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int]),
    "b40c_problem_extract_results_ids64": (c_int, [c_void_p, c_void_p]),
    "b40c_problem_info": (c_int, [c_void_p, POINTER(c_int64), POINTER(c_int64), POINTER(c_void_p),
                                  POINTER(c_void_p), POINTER(c_void_p), POINTER(c_void_p)]),
    "b40c_problem_device": (c_int, [c_void_p, POINTER(c_int)]),
    "b40c_problem_set_stream": (c_int, [c_void_p, c_void_p]),
    "b40c_enactor_create": (c_int, [c_int, c_int, c_int, POINTER(c_void_p)]),
    "b40c_enactor_destroy": (c_int, [c_void_p]),
    "b40c_enactor_frontier_type": (c_int, [c_void_p, POINTER(c_int)]),
    "b40c_enact_search": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int]),
    "b40c_enact_search_async": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int]),
    "b40c_enactor_sync": (c_int, [c_void_p]),
    "b40c_enactor_get_statistics": (c_int, [c_void_p, POINTER(c_longlong), POINTER(c_int), POINTER(c_double)]),
    "b40c_enactor_last_elapsed_ms": (c_int, [c_void_p, POINTER(c_float)]),
    "b40c_enactor_set_stream": (c_int, [c_void_p, c_void_p]),
    "b40c_enactor_set_policy": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    "b40c_enactor_set_level_log": (c_int, [c_void_p, c_int]),
    "b40c_enactor_level_times": (c_int, [c_void_p, c_int, POINTER(c_int64), POINTER(c_int64), POINTER(c_int)]),
    "b40c_enactor_level_log": (c_int, [c_void_p, c_int, POINTER(c_int64), POINTER(c_int), POINTER(c_int),
                                       POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "b40c_enactor_set_direction_optimizing": (c_int, [c_void_p, c_int, c_int]),
    "b40c_enactor_set_wait_limit_us": (c_int, [c_void_p, c_longlong]),
    "b40c_enactor_set_l2_persistence": (c_int, [c_void_p, c_int]),
    "b40c_enactor_set_bottom_up_staging": (c_int, [c_void_p, c_int]),
    "b40c_enactor_set_narrow_levels": (c_int, [c_void_p, c_int, c_int, c_int]),
    "b40c_enactor_narrow_team": (c_int, [c_void_p, POINTER(c_int)]),
    "b40c_graph_grid2d": (c_int, [c_int, c_int, POINTER(CsrT)]),
    "b40c_graph_grid3d": (c_int, [c_int, c_int, POINTER(CsrT)]),
    "b40c_graph_rmat": (c_int, [c_int, c_int, c_double, c_double, c_double, c_uint64, c_int, POINTER(CsrT)]),
    "b40c_graph_erdos_renyi": (c_int, [c_int, c_double, c_uint64, POINTER(CsrT)]),
    "b40c_graph_from_coo": (c_int, [c_int, c_int64, c_void_p, c_void_p, POINTER(CsrT)]),
    "b40c_graph_read_market": (c_int, [c_char_p, c_int, POINTER(CsrT)]),
    "b40c_graph_read_metis": (c_int, [c_char_p, POINTER(CsrT)]),
    "b40c_graph_read_dimacs": (c_int, [c_char_p, c_int, POINTER(CsrT)]),
    "b40c_csr_free": (c_int, [POINTER(CsrT)]),
    "b40c_graph_sample_sources": (c_int, [POINTER(CsrT), c_int, c_uint64, c_void_p]),
    "b40c_debug_barrier_timeout": (c_int, [c_int, c_longlong]),
    "b40c_batch_create": (c_int, [c_int, POINTER(c_void_p)]),
    "b40c_batch_destroy": (c_int, [c_void_p]),
    "b40c_batch_add_graph": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, POINTER(c_int)]),
    "b40c_batch_set_policy": (c_int, [c_void_p, c_int, c_int, c_int, c_int]),
    "b40c_batch_set_stream": (c_int, [c_void_p, c_void_p]),
    "b40c_batch_set_direction_optimizing": (c_int, [c_void_p, c_int, c_int]),
    "b40c_server_set_direction_optimizing": (c_int, [c_void_p, c_int, c_int]),
    "b40c_batch_run": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int]),
    "b40c_batch_run_async": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int]),
    "b40c_batch_sync": (c_int, [c_void_p]),
    "b40c_batch_extract": (c_int, [c_void_p, c_int, c_void_p]),
    "b40c_batch_search_depth": (c_int, [c_void_p, c_int, POINTER(c_int)]),
    "b40c_batch_last_elapsed_ms": (c_int, [c_void_p, POINTER(c_float)]),
    "b40c_server_create": (c_int, [c_int, c_int, c_longlong, POINTER(c_void_p)]),
    "b40c_server_destroy": (c_int, [c_void_p]),
    "b40c_server_add_graph": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, POINTER(c_int)]),
    "b40c_server_set_policy": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_int]),
    "b40c_server_run_trace": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                      POINTER(c_double)]),
    "b40c_server_stats": (c_int, [c_void_p, POINTER(c_longlong), POINTER(c_longlong)]),
    "b40c_enact_search_no_alloc": (c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p, POINTER(c_int),
                                           c_void_p]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Loads libb40c_bfs.so once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m back40computing_b200.build` "
                "(the BFS path has no CPU fallback)")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().b40c_last_error_string()
    return msg.decode() if msg else ""

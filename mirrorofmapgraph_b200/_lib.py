"""ctypes binding of ``lib/libmapgraph_b200.so`` (the C ABI in include/mapgraph_b200.h).

Loading fails loudly when the library is missing: there is no Python or CPU
implementation of the engine to fall back to.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libmapgraph_b200.so")

MG_OK = 0
MG_ERR_ARG = 1
MG_ERR_OOM = 2
MG_ERR_QUEUE_OVERFLOW = 3
MG_ERR_TIMEOUT = 4
MG_ERR_CUDA = 5
MG_ERR_NO_DEVICE = 6
MG_ERR_UNSUPPORTED = 7

MG_DTYPE_NONE, MG_DTYPE_I32, MG_DTYPE_F32 = 0, 1, 2
MG_GRAPH_SYMMETRIC, MG_GRAPH_NO_CSC, MG_GRAPH_DEVICE_INPUT, MG_GRAPH_ASYNC_UPLOAD = 0x1, 0x2, 0x4, 0x8
MG_DIR_AUTO, MG_DIR_PUSH, MG_DIR_PULL = 0, 1, 2
MG_PR_REFCOMPAT, MG_PR_NORMALIZED = 0, 1
MG_W_NONE, MG_W_UNIFORM_INT, MG_W_LOGNORMAL = 0, 1, 2
MG_BFS_NOALLOC_MAX_VERTICES = 1 << 20
MG_BFS_NOALLOC_MAX_SOURCES = 1024


class MgOpts(C.Structure):
    _fields_ = [("directed", C.c_int32), ("iter_num", C.c_int32), ("direction", C.c_int32),
                ("device_output", C.c_int32), ("queue_sizing", C.c_double), ("threshold", C.c_int32),
                ("use_graph", C.c_int32), ("delta", C.c_int32), ("reserved", C.c_int32 * 3)]


class MgStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("edges_traversed", C.c_int64), ("edges_inspected", C.c_int64),
                ("bytes_compulsory", C.c_int64), ("kernel_ms", C.c_double), ("residual", C.c_double),
                ("launches", C.c_int64), ("status_detail", C.c_int32), ("variant", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class MgPrOpts(C.Structure):
    _fields_ = [("mode", C.c_int32), ("directed", C.c_int32), ("max_iter", C.c_int32), ("weighted", C.c_int32),
                ("alpha", C.c_double), ("tol", C.c_double), ("compensated", C.c_int32),
                ("device_output", C.c_int32), ("use_graph", C.c_int32), ("gather_kernel", C.c_int32),
                ("autotune", C.c_int32), ("group_width", C.c_int32), ("seg_hub_edges", C.c_int32),
                ("seg_block_cols", C.c_int32)]


class MgPartLevel(C.Structure):
    _fields_ = [("frontier", C.c_int64), ("frontier_edges", C.c_int64), ("level", C.c_int32),
                ("done", C.c_int32), ("direction", C.c_int32), ("reserved", C.c_int32),
                ("residual", C.c_double)]


class MgLevelRecord(C.Structure):
    _fields_ = [("level", C.c_int32), ("direction", C.c_int32), ("frontier", C.c_int64),
                ("frontier_edges", C.c_int64), ("value", C.c_double), ("time_ns", C.c_uint64)]


MG_TRACE_LEVELS = 4096


class MgTuning(C.Structure):
    _fields_ = [("sssp_heavy", C.c_int32), ("sssp_heavy_small", C.c_int32), ("sssp_ctas_per_sm", C.c_int32),
                ("sssp_chunk_cap", C.c_int32), ("sssp_batch_heavy", C.c_int32), ("bfs_cta_th", C.c_int32),
                ("bfs_grid_th", C.c_int32), ("bfs_defer_warp", C.c_int32), ("bfs_persist_max", C.c_int32),
                ("bfs_persist_edges", C.c_int32), ("bfs_alpha", C.c_int32), ("bfs_beta", C.c_int32),
                ("bfs_sparse_degree", C.c_int32), ("bfs_ctas_per_sm", C.c_int32), ("bfs_tail_max", C.c_int32),
                ("bfs_tail_edges", C.c_int32), ("cc_rounds", C.c_int32), ("reserved", C.c_int32 * 15)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class MgHostCsr(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("row_offsets", C.POINTER(C.c_int32)),
                ("col_idx", C.POINTER(C.c_int32)), ("weights_i32", C.POINTER(C.c_int32)),
                ("weights_f32", C.POINTER(C.c_float))]


# Every symbol the public headers declare, with its ctypes signature.
_P = C.c_void_p
_I32P = C.POINTER(C.c_int32)
_I64P = C.POINTER(C.c_int64)
SIGNATURES = {
    "mg_status_string": (C.c_char_p, [C.c_int]),
    "mg_last_error": (C.c_char_p, []),
    "mg_version": (C.c_char_p, []),
    "mg_device_count": (C.c_int32, []),
    "mg_graph_create": (C.c_int, [_P, _P, _P, C.c_int, C.c_int64, C.c_int64, C.c_uint32, C.POINTER(_P)]),
    "mg_graph_destroy": (C.c_int, [_P]),
    "mg_graph_sync": (C.c_int, [_P]),
    "mg_graph_info": (C.c_int, [_P, _I64P, _I64P, C.POINTER(C.c_uint32), _I32P]),
    "mg_graph_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "mg_graph_device_arrays": (C.c_int, [_P] + [C.POINTER(_P)] * 6),
    "mg_bfs": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_bfs_noalloc": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_bfs_predecessors": (C.c_int, [_P, _P, _P, C.POINTER(MgOpts)]),
    "mg_sssp": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_cc": (C.c_int, [_P, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_pagerank": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(MgPrOpts), C.POINTER(MgStats)]),
    "mg_bfs_batch": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_sssp_batch": (C.c_int, [_P, _P, C.c_int32, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_graph_create_ragged": (C.c_int, [C.c_int32, _P, _P, _P, _P, C.c_uint32, C.POINTER(_P)]),
    "mg_graph_ragged_bases": (C.c_int, [_P, _P]),
    "mg_bfs_ragged": (C.c_int, [_P, _P, _P, C.POINTER(MgOpts), C.POINTER(MgStats)]),
    "mg_pagerank_backward": (C.c_int, [_P, _P, _P, _P, _P, _P, C.POINTER(MgPrOpts), C.POINTER(MgStats)]),
    # host ingest / generators (include/mapgraph_b200_io.h)
    "mg_host_csr_free": (None, [C.POINTER(MgHostCsr)]),
    "mg_gen_er": (C.c_int, [C.c_int64, C.c_int64, C.c_uint64, C.c_int32, C.c_double, C.c_double,
                            C.POINTER(MgHostCsr)]),
    "mg_gen_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int32,
                              C.c_int32, C.c_double, C.c_double, C.POINTER(MgHostCsr)]),
    "mg_gen_lattice": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_uint64, C.c_int32, C.c_double, C.c_double,
                                 C.POINTER(MgHostCsr)]),
    "mg_read_market": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(MgHostCsr)]),
    "mg_write_market": (C.c_int, [C.c_char_p, C.POINTER(MgHostCsr), C.c_int32]),
    "mg_save_csr": (C.c_int, [C.c_char_p, C.POINTER(MgHostCsr)]),
    "mg_load_csr": (C.c_int, [C.c_char_p, C.POINTER(MgHostCsr)]),
    "mg_host_csr_to_csc": (C.c_int, [C.c_int64, C.c_int64, _P, _P, _P, _P, _P]),
    "mg_part_create": (C.c_int, [C.c_int64, C.c_int64, C.c_int64, _P, _P, _P, _P, _P, C.c_uint32,
                                 C.POINTER(_P)]),
    "mg_part_destroy": (C.c_int, [_P]),
    "mg_part_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "mg_part_words": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "mg_part_bfs_begin": (C.c_int, [_P, _P, C.c_int32, C.POINTER(MgOpts), C.POINTER(MgPartLevel)]),
    "mg_part_bfs_step": (C.c_int, [_P, _P]),
    "mg_part_bfs_merge": (C.c_int, [_P, _P, C.c_int32, C.POINTER(MgPartLevel)]),
    "mg_part_bfs_result": (C.c_int, [_P, _P, C.c_int32, C.POINTER(MgStats)]),
    "mg_part_pr_begin": (C.c_int, [_P, C.POINTER(MgPrOpts), C.POINTER(MgPartLevel)]),
    "mg_part_pr_step": (C.c_int, [_P, _P]),
    "mg_part_pr_merge": (C.c_int, [_P, _P, C.c_int32, C.c_int64, _P, C.POINTER(MgPartLevel)]),
    "mg_part_pr_result": (C.c_int, [_P, _P, C.c_int32, C.POINTER(MgStats)]),
    "mg_graph_trace": (C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "mg_tuning_defaults": (None, [C.POINTER(MgTuning)]),
    "mg_graph_degree_stats": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "mg_graph_set_tuning": (C.c_int, [_P, C.POINTER(MgTuning)]),
    "mg_graph_get_tuning": (C.c_int, [_P, C.POINTER(MgTuning)]),
    "mg_debug_fail_alloc": (C.c_int, [C.c_int64]),
    "mg_debug_barrier_skew": (C.c_int, [C.c_int32, C.c_int64]),
    "mg_debug_seg_plan": (C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int64)]),
}

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Loads the engine library (once) and binds every exported symbol."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"mapgraph_b200 engine library not found at {p}; build it with "
            "`python -m mirrorofmapgraph_b200._build` (there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib

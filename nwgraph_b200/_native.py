"""ctypes binding of libnwgpu.so (the C ABI declared in include/nwgpu.h).

Loading fails loudly when the library is missing: the engine has no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnwgpu.so")

# enum nwgpu_status
OK = 0
ERR_INVALID_ARG = 1
ERR_INVALID_GRAPH = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_ABORTED = 5
ERR_NO_DEVICE = 6
ERR_UNSUPPORTED = 7

GRAPH_DEVICE_PTRS = 0x1
GRAPH_TRANSPOSE = 0x2
GRAPH_NO_RELABEL = 0x4
GRAPH_AUTOTUNE = 0x8
NOALLOC_MAX_VERTICES = 1048576
NOALLOC_MAX_ENTRIES = 33554432

MODE_PARITY = 0
LAUNCH_GRAPH = 0
LAUNCH_STREAM = 1

_STATUS_NAMES = {OK: "OK", ERR_INVALID_ARG: "INVALID_ARG", ERR_INVALID_GRAPH: "INVALID_GRAPH", ERR_CUDA: "CUDA",
                 ERR_OUT_OF_MEMORY: "OUT_OF_MEMORY", ERR_ABORTED: "ABORTED", ERR_NO_DEVICE: "NO_DEVICE",
                 ERR_UNSUPPORTED: "UNSUPPORTED"}


class NwgpuError(RuntimeError):
    """A nonzero nwgpu_status; ``.status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"nwgpu {_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class GraphInfo(C.Structure):
    _fields_ = [("n", C.c_uint64), ("nnz", C.c_uint64), ("num_tiles", C.c_uint64), ("tile_items", C.c_uint32),
                ("grid", C.c_uint32), ("device_bytes", C.c_uint64), ("device", C.c_int32),
                ("has_weights", C.c_int32), ("has_transpose", C.c_int32), ("binned", C.c_int32),
                ("sweep_threads", C.c_uint32), ("sweep_grid", C.c_uint32), ("hub_smem_ids", C.c_uint32),
                ("hub_l1_ids", C.c_uint32), ("tuned", C.c_int32), ("tuned_us_per_sweep", C.c_float),
                ("blocked", C.c_int32), ("block_count", C.c_uint32), ("block_items", C.c_uint32),
                ("block_loads", C.c_uint32), ("block_piece_entries", C.c_uint64),
                ("long_row_entries", C.c_uint32), ("chunk_entries", C.c_uint32),
                ("bin0_rows_per_warp", C.c_uint32)]


class PrOptions(C.Structure):
    _fields_ = [("size", C.c_uint32), ("mode", C.c_uint32), ("launch", C.c_uint32), ("device_ptrs", C.c_uint32),
                ("reserved0", C.c_uint32), ("stream", C.c_void_p), ("reserved", C.c_uint32 * 2)]


class PrStats(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("final_error", C.c_double), ("converged", C.c_int32),
                ("device_ms", C.c_double), ("ms_per_iter", C.c_double), ("bytes_per_iter", C.c_double),
                ("gteps", C.c_double), ("errors", C.POINTER(C.c_double)), ("errors_cap", C.c_uint64)]


class PprStats(C.Structure):
    _fields_ = [("iterations", C.c_uint64), ("all_converged", C.c_int32), ("device_ms", C.c_double),
                ("ms_per_iter", C.c_double), ("bytes_per_iter", C.c_double),
                ("col_iterations", C.POINTER(C.c_uint32)), ("col_errors", C.POINTER(C.c_double)),
                ("col_converged", C.POINTER(C.c_int32))]


class BatchStats(C.Structure):
    _fields_ = [("sweeps", C.c_uint64), ("converged_graphs", C.c_uint64), ("device_ms", C.c_double),
                ("entries_swept", C.c_double), ("gteps", C.c_double),
                ("graph_iterations", C.POINTER(C.c_uint32)), ("graph_errors", C.POINTER(C.c_double)),
                ("graph_converged", C.POINTER(C.c_int32))]


FILE_MATRIX_MARKET = 1
FILE_NW_EDGE_LIST = 2
FILE_NW_ADJACENCY = 3


class EdgeFile(C.Structure):
    _fields_ = [("format", C.c_int32), ("directed", C.c_int32), ("has_values", C.c_int32), ("n", C.c_uint64),
                ("max_edges", C.c_uint64)]


# Every symbol include/nwgpu.h declares, with its C signature.
_vp = C.c_void_p
SIGNATURES = {
    "nwgpu_abi_version": (C.c_int, []),
    "nwgpu_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "nwgpu_graph_create": (C.c_int, [_vp, _vp, _vp, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(_vp)]),
    "nwgpu_graph_destroy": (C.c_int, [_vp]),
    "nwgpu_graph_get_info": (C.c_int, [_vp, C.POINTER(GraphInfo)]),
    "nwgpu_pr_run": (C.c_int, [_vp, _vp, _vp, C.c_float, C.c_float, C.c_uint64, C.POINTER(PrOptions),
                               C.POINTER(PrStats)]),
    "nwgpu_pr_residual_run": (C.c_int, [_vp, _vp, _vp, C.c_float, C.c_float, C.c_uint64, C.POINTER(PrOptions),
                                        C.POINTER(PrStats)]),
    "nwgpu_ppr_run": (C.c_int, [_vp, _vp, C.c_uint32, _vp, C.c_float, C.c_float, C.c_uint64, C.POINTER(PrOptions),
                                C.POINTER(PrStats)]),
    "nwgpu_ppr_batched": (C.c_int, [_vp, _vp, _vp, C.c_uint32, _vp, C.c_float, C.c_float, C.c_uint64,
                                    C.POINTER(PrOptions), C.POINTER(PprStats)]),
    "nwgpu_wppr_batched": (C.c_int, [_vp, _vp, C.c_uint32, _vp, C.c_float, C.c_float, C.c_uint64,
                                     C.POINTER(PrOptions), C.POINTER(PprStats)]),
    "nwgpu_ppr_batched_teleports": (C.c_int, [_vp, _vp, _vp, C.c_uint32, _vp, C.c_float, C.c_float, C.c_uint64,
                                              C.POINTER(PrOptions), C.POINTER(PprStats)]),
    "nwgpu_pr_run_noalloc": (C.c_int, [_vp, _vp, C.c_uint64, C.c_uint64, _vp, _vp, C.c_float, C.c_float,
                                       C.c_uint64, _vp, C.POINTER(PrStats)]),
    "nwgpu_abort": (C.c_int, [_vp]),
    "nwgpu_selftest_bounded_wait": (C.c_int, [C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_double)]),
    "nwgpu_spmv": (C.c_int, [_vp, _vp, _vp, C.POINTER(PrOptions)]),
    "nwgpu_release_cached_memory": (C.c_int, []),
    "nwgpu_wpr_run": (C.c_int, [_vp, _vp, _vp, C.c_float, C.c_float, C.c_uint64, C.POINTER(PrOptions),
                                C.POINTER(PrStats)]),
    "nwgpu_pr_vjp": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_float, C.c_float, C.c_uint64, C.POINTER(PrOptions),
                               C.POINTER(PrStats)]),
    "nwgpu_edge_file_probe": (C.c_int, [C.c_char_p, C.POINTER(EdgeFile)]),
    "nwgpu_edge_file_read": (C.c_int, [C.c_char_p, _vp, _vp, _vp, C.c_uint64, C.POINTER(C.c_uint64), C.c_int]),
    "nwgpu_edge_file_write_nw": (C.c_int, [C.c_char_p, _vp, _vp, C.c_uint64, C.c_uint64, C.c_int]),
    "nwgpu_adjacency_file_read": (C.c_int, [C.c_char_p, _vp, _vp, _vp, C.c_uint64, C.c_uint64,
                                            C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "nwgpu_csr_from_edges": (C.c_int, [_vp, _vp, C.c_uint64, C.c_uint64, C.c_uint32, _vp, _vp, C.c_uint64,
                                       C.POINTER(C.c_uint64), _vp, _vp]),
    "nwgpu_rmat_edges": (C.c_int, [C.c_uint32, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_uint64,
                                   C.c_uint64, _vp, _vp, _vp]),
    "nwgpu_grid_edges": (C.c_int, [C.c_uint64, _vp, _vp, _vp]),
    "nwgpu_shard_create": (C.c_int, [_vp, _vp, C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, _vp, C.c_uint64,
                                     C.c_uint32, C.POINTER(_vp)]),
    "nwgpu_shard_destroy": (C.c_int, [_vp]),
    "nwgpu_shard_start": (C.c_int, [_vp, _vp, C.c_int, _vp, _vp]),
    "nwgpu_shard_sweep": (C.c_int, [_vp, _vp, _vp, C.c_float, _vp, _vp]),
    "nwgpu_shard_decide": (C.c_int, [_vp, _vp, C.c_double, C.c_uint64, _vp, _vp, C.c_uint64, _vp]),
    "nwgpu_shard_rank_slice": (C.c_int, [_vp, _vp, _vp]),
    "nwgpu_shard_unpermute": (C.c_int, [_vp, _vp, _vp, _vp]),
    "nwgpu_batch_create": (C.c_int, [C.c_uint64, _vp, _vp, _vp, _vp, C.c_uint32, C.POINTER(_vp)]),
    "nwgpu_batch_destroy": (C.c_int, [_vp]),
    "nwgpu_pr_ragged": (C.c_int, [_vp, _vp, _vp, C.c_float, C.c_float, C.c_uint64, C.POINTER(PrOptions),
                                  C.POINTER(BatchStats)]),
}

_lib = None


def lib():
    """The loaded libnwgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m nwgraph_b200.build` "
                              "(the engine has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().nwgpu_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != OK:
        raise NwgpuError(status, last_error())

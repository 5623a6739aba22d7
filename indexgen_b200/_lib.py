"""ctypes binding of libindexgen_cuda.so (the C ABI in include/indexgen_cuda.h).

The shared object is built in-tree by ``indexgen_b200.build``.  Loading fails
loudly when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libindexgen_cuda.so")

# Every entry point include/indexgen_cuda.h declares.
EXPORTS = (
    "ig_version", "ig_status_string", "ig_ctx_create", "ig_ctx_destroy", "ig_last_error", "ig_ctx_stream",
    "ig_ctx_reserve", "ig_ctx_launches", "ig_ctx_set_profiling", "ig_ctx_phase_time", "ig_pack", "ig_filter", "ig_graph_build", "ig_graph_free",
    "ig_graph_stats", "ig_graph_upper_csr", "ig_graph_pairs", "ig_graph_device_csr", "ig_graph_adjacency",
    "ig_graph_device_adjacency", "ig_graph_codebook",
    "ig_solve", "ig_count_conflicts", "ig_codebook_from_adjacency", "ig_codebook_from_upper_csr", "ig_count_conflicts_noalloc",
    "ig_set_greedy_threads", "ig_greedy_stats",
    "ig_assign_centers", "ig_cluster_solve", "ig_graph_write_adj_list", "ig_graph_read_adj_list",
    "ig_batch_build", "ig_graph_job_count", "ig_graph_job_stats", "ig_graph_job_tiling", "ig_graph_job_codebooks", "ig_solve_batch",
    "ig_server_create", "ig_server_submit", "ig_server_poll", "ig_server_wait", "ig_server_cancel",
    "ig_server_stats", "ig_server_destroy",
    "ig_lane_form", "ig_ctx_autotune", "ig_ctx_set_work_split", "ig_ctx_work_split", "ig_ctx_set_autotune",
    "ig_ctx_set_graphs", "ig_ctx_graph_stats", "ig_ctx_set_coalescing", "ig_ctx_coalesce_stats",
    "ig_ctx_set_wait_limit", "ig_ctx_inject_fault", "ig_ctx_set_host_budget", "ig_ctx_host_budget", "ig_ctx_alloc_stats", "ig_ctx_set_host_lists",
)

STATUS = {0: "IG_OK", 1: "IG_ERR_INPUT", 2: "IG_ERR_CAPACITY", 3: "IG_ERR_OOM", 4: "IG_ERR_CUDA",
          5: "IG_ERR_TIMEOUT", 6: "IG_ERR_CANCELLED", 7: "IG_ERR_STATE"}


class IndexGenError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        self.code = STATUS.get(status, str(status))
        super().__init__(f"{where}: {self.code}" + (f" ({detail})" if detail else ""))


_lib = None


class ServerOpts(ctypes.Structure):
    """ig_server_opts of include/indexgen_cuda.h."""

    _fields_ = [("host_threads", ctypes.c_int), ("max_batch_jobs", ctypes.c_int), ("order_threads", ctypes.c_int),
                ("reserved", ctypes.c_int), ("max_batch_pairs", ctypes.c_int64),
                ("hbm_budget_bytes", ctypes.c_int64), ("pool_reserve_bytes", ctypes.c_int64)]


_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_int = ctypes.c_int


def _declare(L):
    sig = {
        "ig_version": (ctypes.c_char_p, []),
        "ig_status_string": (ctypes.c_char_p, [_int]),
        "ig_ctx_create": (_int, [ctypes.POINTER(_vp), _int]),
        "ig_ctx_destroy": (_int, [_vp]),
        "ig_last_error": (ctypes.c_char_p, [_vp]),
        "ig_ctx_stream": (_int, [_vp, ctypes.POINTER(_vp)]),
        "ig_ctx_reserve": (_int, [_vp, _i64]),
        "ig_ctx_launches": (_i64, [_vp]),
        "ig_ctx_set_profiling": (_int, [_vp, _int]),
        "ig_ctx_phase_time": (_int, [_vp, _int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i64)]),
        "ig_pack": (_int, [ctypes.c_char_p, _i64, _int, _i64, _vp, ctypes.POINTER(_i64)]),
        "ig_filter": (_int, [_vp, _i64, _int, _int, ctypes.c_double, ctypes.c_double, _vp]),
        "ig_graph_build": (_int, [_vp, _vp, _i32, _int, _int, _int, ctypes.POINTER(_vp)]),
        "ig_graph_free": (_int, [_vp]),
        "ig_graph_stats": (_int, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(_i64)]),
        "ig_graph_upper_csr": (_int, [_vp, _vp, _vp]),
        "ig_graph_pairs": (_int, [_vp, _vp]),
        "ig_graph_device_csr": (_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
        "ig_graph_adjacency": (_int, [_vp, _vp, _vp]),
        "ig_graph_device_adjacency": (_int, [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)]),
        "ig_graph_codebook": (_int, [_vp, _int, _vp, ctypes.POINTER(_i32)]),
        "ig_solve": (_int, [_vp, _vp, _i32, _int, _int, _int, _vp, ctypes.POINTER(_i32), ctypes.POINTER(_i64)]),
        "ig_count_conflicts": (_int, [_vp, _vp, _i32, _int, _int, ctypes.POINTER(_i64)]),
        "ig_codebook_from_upper_csr": (_int, [_vp, _vp, _i32, _int, _vp, ctypes.POINTER(_i32)]),
        "ig_codebook_from_adjacency": (_int, [_vp, _vp, _i32, _vp, ctypes.POINTER(_i32)]),
        "ig_set_greedy_threads": (_int, [_int, _i64]),
        "ig_greedy_stats": (_int, [ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
        "ig_count_conflicts_noalloc": (_int, [_vp, _i32, _int, _int, _vp, _vp]),
        "ig_assign_centers": (_int, [_vp, _vp, _i64, _vp, _i32, _int, _int, _vp]),
        "ig_graph_write_adj_list": (_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_i64)]),
        "ig_graph_read_adj_list": (_int, [_vp, ctypes.c_char_p, ctypes.POINTER(_vp)]),
        "ig_cluster_solve": (_int, [_vp, _vp, _i32, _int, _int, _i32, _i32, ctypes.c_uint64, _i32, _int, _vp,
                                    ctypes.POINTER(_i32), ctypes.POINTER(_i32), _vp]),
        "ig_batch_build": (_int, [_vp, _vp, _vp, _i32, _vp, _vp, _int, ctypes.POINTER(_vp)]),
        "ig_graph_job_count": (_int, [_vp, ctypes.POINTER(_i32)]),
        "ig_graph_job_stats": (_int, [_vp, _i32, ctypes.POINTER(_i64), ctypes.POINTER(_i32), ctypes.POINTER(_i64)]),
        "ig_graph_job_tiling": (_int, [_vp, _i32, ctypes.POINTER(_i32), ctypes.POINTER(_i32)]),
        "ig_graph_job_codebooks": (_int, [_vp, _int, _int, _vp, _vp]),
        "ig_solve_batch": (_int, [_vp, _vp, _vp, _i32, _vp, _vp, _int, _int, _vp, _vp, _vp]),
        "ig_server_create": (_int, [_vp, ctypes.POINTER(ServerOpts), ctypes.POINTER(_vp)]),
        "ig_server_submit": (_int, [_vp, _vp, _i32, _int, _int, ctypes.POINTER(_i64)]),
        "ig_server_poll": (_int, [_vp, _i64, ctypes.POINTER(_int)]),
        "ig_server_wait": (_int, [_vp, _i64, _vp, ctypes.POINTER(_i32), ctypes.POINTER(_i64),
                                  ctypes.POINTER(ctypes.c_double)]),
        "ig_server_cancel": (_int, [_vp, _i64]),
        "ig_server_stats": (_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
        "ig_server_destroy": (_int, [_vp]),
        "ig_lane_form": (_int, [_int, _int]),
        "ig_ctx_autotune": (_int, [_vp, _vp, _i32, _int, _int, _int, ctypes.POINTER(_i32)]),
        "ig_ctx_set_work_split": (_int, [_vp, _int, _i32]),
        "ig_ctx_work_split": (_int, [_vp, _int, ctypes.POINTER(_i32), ctypes.POINTER(_int)]),
        "ig_ctx_set_autotune": (_int, [_vp, _int]),
        "ig_ctx_set_graphs": (_int, [_vp, _int]),
        "ig_ctx_graph_stats": (_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
        "ig_ctx_set_coalescing": (_int, [_vp, _int]),
        "ig_ctx_set_wait_limit": (_int, [_vp, _i64]),
        "ig_ctx_set_host_budget": (_int, [_vp, _i64]),
        "ig_ctx_alloc_stats": (_int, [_vp, ctypes.POINTER(_i64)]),
        "ig_ctx_set_host_lists": (_int, [_vp, _int]),
        "ig_ctx_host_budget": (_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
        "ig_ctx_inject_fault": (_int, [_vp, _int, _i64]),
        "ig_ctx_coalesce_stats": (_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def lib():
    """Load libindexgen_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m indexgen_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def check(status: int, where: str, ctx=None):
    if status != 0:
        detail = ""
        if ctx:
            msg = lib().ig_last_error(ctx)
            detail = msg.decode() if msg else ""
        raise IndexGenError(status, where, detail)


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0

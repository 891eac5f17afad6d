"""ctypes binding of libartea_gpu.so (the C-ABI declared in include/artea_gpu.h).

The library is built in-tree (``artea_b200/lib/libartea_gpu.so``) by
``artea_b200.build``; importing this module never falls back to anything
else: if the library is missing, every entry point raises.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_int, c_uint32, c_uint64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libartea_gpu.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "artea_gpu.h")

OK, EINVAL, ENOMEM, ECUDA, EGRAPH, EIO, EKERNEL, ETIMEOUT, ENODEV, EBUSY = range(10)
STATUS_NAMES = {OK: "OK", EINVAL: "EINVAL", ENOMEM: "ENOMEM", ECUDA: "ECUDA", EGRAPH: "EGRAPH", EIO: "EIO",
                EKERNEL: "EKERNEL", ETIMEOUT: "ETIMEOUT", ENODEV: "ENODEV", EBUSY: "EBUSY"}

METRIC_EUCLIDEAN_SQR, METRIC_EUCLIDEAN, METRIC_COSINE, METRIC_DOT = 0, 1, 2, 3
MODE_EXACT, MODE_FAST = 0, 1
SCHEDULE_AUTO, SCHEDULE_PLAIN, SCHEDULE_PERSISTENT = 0, 1, 2


class GraphDesc(ctypes.Structure):
    _fields_ = [
        ("num_vertices", c_uint32),
        ("top_level", c_uint32),
        ("ul_max_nbr_size", c_uint32),
        ("bl_max_nbr_size", c_uint32),
        ("entry_point_vid", c_uint32),
        ("vertex_info", POINTER(c_uint32)),
        ("group_offsets", POINTER(POINTER(c_uint64))),
        ("group_sizes", POINTER(c_uint64)),
        ("neighbor_ids", POINTER(c_uint32)),
        ("num_neighbor_ids", c_uint64),
    ]


class HgraInfo(ctypes.Structure):
    _fields_ = [
        ("num_vertices", c_uint32),
        ("top_level", c_uint32),
        ("ul_max_nbr_size", c_uint32),
        ("bl_max_nbr_size", c_uint32),
        ("entry_point_vid", c_uint32),
        ("num_groups", c_uint32),
        ("num_neighbor_ids", c_uint64),
        ("num_offsets", c_uint64),
        ("group_sizes", c_uint64 * 64),
    ]


class QueryStats(ctypes.Structure):
    _fields_ = [
        ("dist_evals", c_uint32),
        ("upper_rows", c_uint32),
        ("upper_row_ids", c_uint32),
        ("l0_rows", c_uint32),
        ("l0_row_ids", c_uint32),
        ("upper_dist_evals", c_uint32),
        ("results", c_uint32),
        ("visited_spills", c_uint32),
    ]


class RouterOpts(ctypes.Structure):
    _fields_ = [
        ("metric", c_int),
        ("mode", c_int),
        ("schedule", c_int),
        ("warps_per_cta", c_uint32),
        ("ctas_per_sm", c_uint32),
        ("max_batch", c_uint32),
        ("max_queue", c_uint32),
        ("use_graphs", c_uint32),
        ("visited_hash_bits", c_uint32),
        ("register_budget", c_uint32),
        ("stage_rows", c_uint32),
        ("pipeline", c_uint32),
        ("prefetch_rows", c_uint32),
        ("order_queries", c_uint32),
        ("warps_per_query", c_uint32),
        ("queue_slack", c_uint32),
    ]


class ProbeResult(ctypes.Structure):
    _fields_ = [
        ("search_ms", ctypes.c_float),
        ("greedy_ms", ctypes.c_float),
        ("gather_ms", ctypes.c_float),
        ("visited_ms", ctypes.c_float),
        ("queue_ms", ctypes.c_float),
        ("capped_queries", c_uint32),
        ("candidates", c_uint64),
        ("expansions", c_uint64),
        ("gather_mismatches", c_uint32),
        ("visited_mismatches", c_uint32),
        ("queue_mismatches", c_uint32),
    ]


class ServerOpts(ctypes.Structure):
    _fields_ = [
        ("metric", c_int),
        ("mode", c_int),
        ("max_topk", c_uint32),
        ("max_queue", c_uint32),
        ("ring_slots", c_uint32),
        ("warps_per_cta", c_uint32),
        ("idle_polls", c_uint32),
        ("heartbeat_ms", c_uint32),
    ]


# Every exported function with its ctypes signature; the names are exactly
# the functions include/artea_gpu.h declares.
SIGNATURES = {
    "artea_gpu_version": (c_char_p, []),
    "artea_gpu_last_error": (c_char_p, []),
    "artea_gpu_device_count": (c_int, [POINTER(c_int)]),
    "artea_gpu_hgra_probe": (c_int, [c_char_p, POINTER(HgraInfo)]),
    "artea_gpu_hgra_read": (c_int, [c_char_p, c_void_p, c_void_p, c_void_p]),
    "artea_gpu_hgra_write": (c_int, [c_char_p, POINTER(GraphDesc)]),
    "artea_gpu_graph_validate": (c_int, [POINTER(GraphDesc)]),
    "artea_gpu_index_create": (c_int, [POINTER(GraphDesc), c_void_p, c_uint32, c_uint32, c_int, POINTER(c_void_p)]),
    "artea_gpu_index_create_from_hgra": (c_int, [c_char_p, c_void_p, c_uint32, c_uint32, c_int, POINTER(c_void_p)]),
    "artea_gpu_index_download": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "artea_gpu_index_destroy": (c_int, [c_void_p]),
    "artea_gpu_index_bytes": (c_int, [c_void_p, POINTER(c_uint64)]),
    "artea_gpu_router_create": (c_int, [c_void_p, c_uint32, c_uint32, POINTER(RouterOpts), POINTER(c_void_p)]),
    "artea_gpu_router_destroy": (c_int, [c_void_p]),
    "artea_gpu_batch_query": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_uint32, c_void_p,
                                      c_void_p]),
    "artea_gpu_batch_query_device": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_uint32, c_void_p,
                                             c_void_p, c_void_p]),
    "artea_gpu_batch_query_l0_only": (c_int, [c_void_p, c_void_p, c_uint32, c_uint32, c_void_p, c_void_p]),
    "artea_gpu_router_sync": (c_int, [c_void_p]),
    "artea_gpu_router_launches": (c_int, [c_void_p, POINTER(c_uint64)]),
    "artea_gpu_router_last_reruns": (c_int, [c_void_p, POINTER(c_uint32)]),
    "artea_gpu_subsystem_probe": (c_int, [c_void_p, c_int, c_int, c_uint32, c_uint32, c_void_p, c_uint32, c_uint32,
                                          POINTER(ProbeResult)]),
    "artea_gpu_router_set_phase_buffer": (c_int, [c_void_p, c_void_p]),
    "artea_gpu_router_set_early_stop": (c_int, [c_void_p, c_void_p, c_uint32]),
    "artea_gpu_bruteforce": (c_int, [c_void_p, c_int, c_void_p, c_uint32, c_uint32, c_void_p, c_uint32, c_void_p]),
    "artea_gpu_centroid_entry": (c_int, [c_void_p, c_int, c_void_p, c_uint32, c_void_p]),
    "artea_gpu_bruteforce_device": (c_int, [c_void_p, c_int, c_void_p, c_uint32, c_uint32, c_void_p, c_uint32,
                                            c_void_p, c_void_p]),
    "artea_gpu_server_create": (c_int, [c_void_p, POINTER(ServerOpts), POINTER(c_void_p)]),
    "artea_gpu_server_submit": (c_int, [c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, POINTER(c_uint64)]),
    "artea_gpu_server_poll": (c_int, [c_void_p, c_uint64, c_uint32, c_uint32, c_void_p, POINTER(c_int)]),
    "artea_gpu_server_stats": (c_int, [c_void_p, POINTER(c_uint64), POINTER(c_uint64), POINTER(c_uint64)]),
    "artea_gpu_server_destroy": (c_int, [c_void_p]),
    "artea_gpu_server_pause_heartbeat": (c_int, [c_void_p]),
    "artea_gpu_batch_query_noalloc": (c_int, [c_void_p, c_int, c_int, c_uint32, c_uint32, c_void_p, c_uint32, c_uint32,
                                              c_void_p, c_void_p]),
    "artea_gpu_router_tuning": (c_int, [c_void_p, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32),
                                        POINTER(c_uint32)]),
    "artea_gpu_router_tuning_ext": (c_int, [c_void_p, POINTER(c_uint32), POINTER(c_uint32), POINTER(c_uint32),
                                            POINTER(c_uint32), POINTER(c_uint32)]),
}


class ArteaGpuError(RuntimeError):
    """A non-OK status from the C-ABI; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None


def lib() -> ctypes.CDLL:
    """Load libartea_gpu.so once; raise if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run artea_b200.build.build() (nvcc, sm_100a)")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int) -> None:
    if status != OK:
        msg = lib().artea_gpu_last_error().decode(errors="replace")
        raise ArteaGpuError(status, msg)


def ptr(a) -> c_void_p:
    """Raw address of a numpy array, a torch tensor, or None."""
    if a is None:
        return c_void_p(None)
    if hasattr(a, "data_ptr"):
        return c_void_p(a.data_ptr())
    return c_void_p(a.ctypes.data)

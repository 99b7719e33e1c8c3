"""ctypes binding of libsbfs.so (include/sbfs.h).

The library is loaded from ``sbfs/_lib/libsbfs.so`` inside this package (or
from the path in the ``SBFS_LIB`` environment variable); there is no
fallback: if the library is missing or cannot be loaded, every call raises
``NativeUnavailable``.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
# SBFS_LIB may name another build of the same library (e.g. an installed copy)
LIB_PATH = os.environ.get("SBFS_LIB") or os.path.join(HERE, "_lib", "libsbfs.so")

# every symbol include/sbfs.h declares (checked by the CPU test suite)
EXPORTS = [
    "sbfs_abi_version", "sbfs_config_default", "sbfs_create", "sbfs_destroy", "sbfs_last_error",
    "sbfs_status_string", "sbfs_best_parallelism", "sbfs_solve_batch", "sbfs_verify_batch",
    "sbfs_solve_plain", "sbfs_solve_batch_device", "sbfs_device_wait", "sbfs_host_alloc",
    "sbfs_host_free", "sbfs_word_stride", "sbfs_describe_plan", "sbfs_solve_small_noalloc",
    "sbfs_server_config_default", "sbfs_server_start", "sbfs_server_submit", "sbfs_server_submit_many",
    "sbfs_server_poll",
    "sbfs_server_cancel", "sbfs_server_stats_get", "sbfs_server_reset_peak", "sbfs_server_stop",
    "sbfs_generate_reference_batch", "sbfs_dotnet_random_next",
]

STATUS = {0: "SBFS_OK", 1: "SBFS_EINVAL", 2: "SBFS_ENOMEM", 3: "SBFS_ETIMEOUT", 4: "SBFS_ECUDA",
          5: "SBFS_EBUSY", 6: "SBFS_ENOTFOUND", 7: "SBFS_ECANCELED", 8: "SBFS_ESTOPPED"}


class NativeUnavailable(RuntimeError):
    pass


class SbfsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Config(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("slack", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("autotune", ctypes.c_int32),
        ("slots_per_warp", ctypes.c_int32),
        ("warps_per_cta", ctypes.c_int32),
        ("queue_smem", ctypes.c_int32),
        ("chunk", ctypes.c_int32),
        ("small_kernel", ctypes.c_int32),
        ("lane_ring", ctypes.c_int32),
        ("lane_refill", ctypes.c_int32),
        ("lane_warps", ctypes.c_int32),
        ("lane_tail", ctypes.c_int32),
        ("streams", ctypes.c_int32),
        ("level_arena_bytes", ctypes.c_int64),
        ("tune_cache", ctypes.c_char_p),
        ("wait_polls", ctypes.c_int32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("automata", ctypes.c_int64),
        ("expanded", ctypes.c_int64),
        ("synchronizing", ctypes.c_int64),
        ("h2d_bytes", ctypes.c_int64),
        ("d2h_bytes", ctypes.c_int64),
        ("launches", ctypes.c_int32),
        ("classes", ctypes.c_int32),
        ("kernel_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("escalated", ctypes.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("max_batch", ctypes.c_int32),
        ("max_levels", ctypes.c_int32),
        ("queue_capacity", ctypes.c_int32),
        ("arena_bytes", ctypes.c_int64),
        ("small_budget_bytes", ctypes.c_int64),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("id", ctypes.c_uint64),
        ("status", ctypes.c_int32),
        ("len", ctypes.c_int32),
        ("n", ctypes.c_int32),
        ("pad", ctypes.c_int32),
        ("word", ctypes.c_uint64 * 12),
        ("submit_ms", ctypes.c_double),
        ("done_ms", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in (
        "submitted", "completed", "rejected", "cancelled", "pending", "in_flight", "small_batches",
        "level_launches", "arena_used", "arena_peak", "arena_capacity")] + [("now_ms", ctypes.c_double)] + [
        (k, ctypes.c_int64) for k in ("small_used", "small_peak", "small_capacity")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib: Optional[ctypes.CDLL] = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libsbfs.so and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NativeUnavailable(f"{path} is not built (run build.py or __graft_entry__.build())")
    try:
        L = ctypes.CDLL(path)
    except OSError as e:
        raise NativeUnavailable(f"cannot load {path}: {e}") from e
    P = ctypes.c_void_p
    i32, i64 = ctypes.c_int32, ctypes.c_int64
    L.sbfs_abi_version.restype = i32
    L.sbfs_config_default.argtypes = [ctypes.POINTER(Config)]
    L.sbfs_config_default.restype = ctypes.c_int
    L.sbfs_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(P)]
    L.sbfs_create.restype = ctypes.c_int
    L.sbfs_destroy.argtypes = [P]
    L.sbfs_destroy.restype = ctypes.c_int
    L.sbfs_last_error.argtypes = [P]
    L.sbfs_last_error.restype = ctypes.c_char_p
    L.sbfs_status_string.argtypes = [ctypes.c_int]
    L.sbfs_status_string.restype = ctypes.c_char_p
    L.sbfs_best_parallelism.argtypes = [P]
    L.sbfs_best_parallelism.restype = i32
    L.sbfs_word_stride.argtypes = [i32]
    L.sbfs_word_stride.restype = i32
    solve_args = [P, P, i32, P, i32, i64, P, P, i32, ctypes.POINTER(i64), ctypes.POINTER(Stats)]
    for name in ("sbfs_solve_batch", "sbfs_solve_plain"):
        getattr(L, name).argtypes = solve_args
        getattr(L, name).restype = ctypes.c_int
    L.sbfs_verify_batch.argtypes = [P, P, i32, P, i32, i64, P, ctypes.POINTER(i64), ctypes.POINTER(Stats)]
    L.sbfs_verify_batch.restype = ctypes.c_int
    L.sbfs_solve_batch_device.argtypes = [P, P, i32, P, i32, i32, i64, P, P, i32, P, P]
    L.sbfs_solve_batch_device.restype = ctypes.c_int
    L.sbfs_device_wait.argtypes = [P, ctypes.POINTER(Stats)]
    L.sbfs_device_wait.restype = ctypes.c_int
    L.sbfs_host_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(P)]
    L.sbfs_host_alloc.restype = ctypes.c_int
    L.sbfs_solve_small_noalloc.argtypes = [P, i32, i32, i64, P, P, i32, P, P]
    L.sbfs_solve_small_noalloc.restype = ctypes.c_int
    L.sbfs_server_config_default.argtypes = [ctypes.POINTER(ServerConfig)]
    L.sbfs_server_config_default.restype = ctypes.c_int
    L.sbfs_server_start.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(P)]
    L.sbfs_server_start.restype = ctypes.c_int
    L.sbfs_server_submit.argtypes = [P, P, P, i32, ctypes.POINTER(ctypes.c_uint64)]
    L.sbfs_server_submit.restype = ctypes.c_int
    L.sbfs_server_submit_many.argtypes = [P, P, i32, P, i64, P]
    L.sbfs_server_submit_many.restype = ctypes.c_int
    L.sbfs_server_poll.argtypes = [P, ctypes.POINTER(Result), i32, ctypes.POINTER(i32), i32]
    L.sbfs_server_poll.restype = ctypes.c_int
    L.sbfs_server_cancel.argtypes = [P, ctypes.c_uint64]
    L.sbfs_server_cancel.restype = ctypes.c_int
    L.sbfs_server_stats_get.argtypes = [P, ctypes.POINTER(ServerStats)]
    L.sbfs_server_stats_get.restype = ctypes.c_int
    L.sbfs_server_reset_peak.argtypes = [P]
    L.sbfs_server_reset_peak.restype = ctypes.c_int
    L.sbfs_server_stop.argtypes = [P]
    L.sbfs_server_stop.restype = ctypes.c_int
    L.sbfs_describe_plan.argtypes = [P, ctypes.c_char_p, i32]
    L.sbfs_describe_plan.restype = i32
    L.sbfs_host_free.argtypes = [P]
    L.sbfs_host_free.restype = ctypes.c_int
    L.sbfs_generate_reference_batch.argtypes = [i64, i32, i32, P, i32]
    L.sbfs_generate_reference_batch.restype = ctypes.c_int
    L.sbfs_dotnet_random_next.argtypes = [i32, i32, P]
    L.sbfs_dotnet_random_next.restype = ctypes.c_int
    _lib = L
    return L


def check(handle, status: int):
    if status != 0:
        msg = load().sbfs_last_error(handle)
        raise SbfsError(status, msg.decode() if msg else "")

"""Serving front end: a request loop on the GPU (sbfs_server_* in include/sbfs.h).

Requests are single automata.  Those with n <= 20 are gathered into
mini-batches (several in flight) whose kernels deliver each result as soon as
its own search ends; larger ones are admitted into device-resident BFS slots as
their 2^n-bit bitmap and queue fit the memory budget, and advance level by level
alongside every other admitted request (continuous batching).
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional

import numpy as np

from . import _native


RESULT_DTYPE = np.dtype([("id", np.uint64), ("status", np.int32), ("len", np.int32), ("n", np.int32),
                         ("pad", np.int32), ("word", np.uint64, (12,)), ("submit_ms", np.float64),
                         ("done_ms", np.float64)])


class Server:
    def __init__(self, device: int = -1, max_batch: int = 0, max_levels: int = 0, queue_capacity: int = 0,
                 arena_bytes: int = 0, small_budget_bytes: int = 0):
        self.lib = _native.load()
        cfg = _native.ServerConfig()
        self.lib.sbfs_server_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.max_batch = max_batch
        cfg.max_levels = max_levels
        cfg.queue_capacity = queue_capacity
        cfg.arena_bytes = arena_bytes
        cfg.small_budget_bytes = small_budget_bytes
        h = ctypes.c_void_p()
        st = self.lib.sbfs_server_start(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise _native.SbfsError(st, "server start failed")
        self.handle = h
        self._buf = (_native.Result * 4096)()

    def submit(self, a, b, n: int) -> int:
        """Returns the request id; raises SbfsError (EINVAL / EBUSY)."""
        a = np.ascontiguousarray(a[:n], dtype=np.uint8)
        b = np.ascontiguousarray(b[:n], dtype=np.uint8)
        rid = ctypes.c_uint64()
        st = self.lib.sbfs_server_submit(self.handle, a.ctypes.data_as(ctypes.c_void_p),
                                         b.ctypes.data_as(ctypes.c_void_p), n, ctypes.byref(rid))
        if st != 0:
            raise _native.SbfsError(st, "submit refused")
        return rid.value

    def submit_record(self, rec, n: int, lstride: int = 32) -> int:
        return self.submit(rec[:n], rec[lstride:lstride + n], n)

    def submit_many(self, recs, ns, lstride: int = 32) -> np.ndarray:
        """Submits every record in one call (all admitted or none); returns
        their ids.  Raises SbfsError (EINVAL / EBUSY)."""
        recs = np.ascontiguousarray(recs, dtype=np.uint8)
        ns = np.ascontiguousarray(ns, dtype=np.uint8)
        count = int(ns.shape[0])
        if recs.shape != (count, 2 * lstride):
            raise ValueError(f"records must have shape ({count}, {2 * lstride})")
        ids = np.empty(count, dtype=np.uint64)
        st = self.lib.sbfs_server_submit_many(self.handle, recs.ctypes.data_as(ctypes.c_void_p), lstride,
                                              ns.ctypes.data_as(ctypes.c_void_p), count,
                                              ids.ctypes.data_as(ctypes.c_void_p))
        if st != 0:
            raise _native.SbfsError(st, "submit_many refused")
        return ids

    def poll(self, timeout_ms: int = 0, max_results: int = 4096) -> List[dict]:
        got = ctypes.c_int32()
        self.lib.sbfs_server_poll(self.handle, self._buf, min(max_results, len(self._buf)), ctypes.byref(got),
                                  int(timeout_ms))
        out = []
        for i in range(got.value):
            r = self._buf[i]
            out.append({"id": r.id, "status": r.status, "len": r.len, "n": r.n,
                        "word": np.array(r.word[:], dtype=np.uint64), "submit_ms": r.submit_ms,
                        "done_ms": r.done_ms})
        return out

    def poll_array(self, timeout_ms: int = 0, max_results: int = 4096) -> np.ndarray:
        """Like poll, as one structured array (fields of sbfs_result) -- cheap
        for clients that collect many results."""
        got = ctypes.c_int32()
        self.lib.sbfs_server_poll(self.handle, self._buf, min(max_results, len(self._buf)), ctypes.byref(got),
                                  int(timeout_ms))
        return np.frombuffer(self._buf, dtype=RESULT_DTYPE, count=got.value).copy()

    def wait_all(self, ids, timeout_s: float = 120.0) -> Dict[int, dict]:
        import time
        want = set(ids)
        res: Dict[int, dict] = {}
        t_end = time.monotonic() + timeout_s
        while want - res.keys():
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(want - res.keys())} requests unfinished")
            for r in self.poll(timeout_ms=50):
                res[r["id"]] = r
        return res

    def cancel(self, rid: int) -> bool:
        return self.lib.sbfs_server_cancel(self.handle, rid) == 0

    def stats(self) -> dict:
        st = _native.ServerStats()
        self.lib.sbfs_server_stats_get(self.handle, ctypes.byref(st))
        return st.as_dict()

    def reset_peak(self):
        self.lib.sbfs_server_reset_peak(self.handle)

    def stop(self):
        if getattr(self, "handle", None):
            self.lib.sbfs_server_stop(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass

"""ctypes wrapper of liboracle.so, the CPU restatement of the reference's BFS.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU legs, as the checker or the timed CPU baseline.  The product
library never loads it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "sbfs_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        L.orc_solve.argtypes = [P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int64, P, P,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int, P, P]
        L.orc_solve.restype = ctypes.c_int
        L.orc_verify4.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int64, P,
                                  ctypes.c_int, ctypes.c_int, P, P]
        L.orc_verify4.restype = ctypes.c_int
        L.orc_replay.argtypes = [P, ctypes.c_int, P, ctypes.c_int, ctypes.c_int64, P, P,
                                 ctypes.c_int, P]
        L.orc_replay.restype = ctypes.c_int64
        L.orc_fill_array_of_problems.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_int32, P,
                                                 ctypes.c_int, ctypes.c_int]
        L.orc_fill_array_of_problems.restype = ctypes.c_int
        L.orc_dotnet_random_next.argtypes = [ctypes.c_int32, ctypes.c_int32, P]
        L.orc_dotnet_random_next.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def word_stride_for(max_n: int) -> int:
    """u64 words per automaton that hold a word of length (n-1)^2."""
    return max(1, ((max_n - 1) ** 2 + 63) // 64)


def solve(recs: np.ndarray, ns=None, n: int = 0, lstride: int = 32, words: bool = True,
          word_stride: Optional[int] = None, slack: int = 0, threads: int = 1):
    """SlimCPUUntweaked semantics.  Returns dict(len, words, first_violation, expanded)."""
    recs = np.ascontiguousarray(recs, dtype=np.uint8)
    count = recs.shape[0]
    ns_arr = None if ns is None else np.ascontiguousarray(ns, dtype=np.uint8)
    max_n = int(ns_arr.max()) if (ns_arr is not None and count) else int(n)
    out_len = np.empty(count, dtype=np.int32)
    ws = word_stride or word_stride_for(max(max_n, 2))
    out_words = np.zeros((count, ws), dtype=np.uint64) if words else None
    fv = ctypes.c_int64(-1)
    ex = ctypes.c_int64(0)
    st = lib().orc_solve(_ptr(recs), lstride, _ptr(ns_arr), int(n), count, _ptr(out_len),
                         _ptr(out_words), ws if words else 0, slack, threads,
                         ctypes.byref(fv), ctypes.byref(ex))
    if st != 0:
        raise ValueError(f"oracle orc_solve failed with status {st}")
    return {"len": out_len, "words": out_words, "word_stride": ws,
            "first_violation": fv.value, "expanded": ex.value}


def verify4(recs: np.ndarray, n: int, lstride: int, write_len: bool = False, slack: int = 0,
            threads: int = 1):
    """SlimCPU4bits13 semantics (nibble table, Verify mode)."""
    recs = np.ascontiguousarray(recs, dtype=np.uint8)
    count = recs.shape[0]
    out_len = np.empty(count, dtype=np.int32) if write_len else None
    fv = ctypes.c_int64(-1)
    ex = ctypes.c_int64(0)
    st = lib().orc_verify4(_ptr(recs), lstride, n, count, _ptr(out_len), slack, threads,
                           ctypes.byref(fv), ctypes.byref(ex))
    if st != 0:
        raise ValueError(f"oracle orc_verify4 failed with status {st}")
    return {"len": out_len, "first_violation": fv.value, "expanded": ex.value}


def replay(recs: np.ndarray, lens: np.ndarray, words: np.ndarray, ns=None, n: int = 0,
           lstride: int = 32):
    """Verify.cs checks; returns (bad_count, ok_bits)."""
    recs = np.ascontiguousarray(recs, dtype=np.uint8)
    lens = np.ascontiguousarray(lens, dtype=np.int32)
    words = np.ascontiguousarray(words, dtype=np.uint64)
    ns_arr = None if ns is None else np.ascontiguousarray(ns, dtype=np.uint8)
    ok = np.empty(recs.shape[0], dtype=np.uint8)
    bad = lib().orc_replay(_ptr(recs), lstride, _ptr(ns_arr), int(n), recs.shape[0],
                           _ptr(lens), _ptr(words), words.shape[1], _ptr(ok))
    return int(bad), ok


def fill_array_of_problems(count: int, n: int, seed: int, lstride: int = 32, threads: int = 1) -> np.ndarray:
    """Problem.FillArrayOfProblems (SharedDefinitions/Problem.cs:32-58) with
    .NET System.Random, as records of 2*lstride bytes (a = rec[:n],
    b = rec[lstride:lstride + n]); the CPU legs build the reference's batches
    with it so that they never load the product library."""
    count, n, lstride = int(count), int(n), int(lstride)
    out = np.empty((count, 2 * lstride), dtype=np.uint8)
    st = lib().orc_fill_array_of_problems(count, n, int(seed), _ptr(out) if count else None, lstride,
                                          int(threads))
    if st != 0:
        raise ValueError(f"oracle orc_fill_array_of_problems failed with status {st}")
    return out


def dotnet_random_next(seed: int, count: int) -> np.ndarray:
    """The first ``count`` values of ``new System.Random(seed).Next()``."""
    out = np.empty(int(count), dtype=np.int32)
    st = lib().orc_dotnet_random_next(int(seed), int(count), _ptr(out) if count else None)
    if st != 0:
        raise ValueError(f"oracle orc_dotnet_random_next failed with status {st}")
    return out

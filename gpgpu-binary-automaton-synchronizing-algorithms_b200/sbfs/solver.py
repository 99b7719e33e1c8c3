"""Host-side mirror of the reference's solver plugin contract over the C ABI.

``Engine`` owns one ``sbfs_handle`` (include/sbfs.h) and works on packed numpy
records.  ``SlimGPUNative`` implements the reference interface
``IComputable`` (GPGPU/Interfaces/IComputable.cs:11-20) on ``Problem`` /
``ComputationResult`` objects, with the same argument meaning:

  Compute(problems, problemsReadingIndex, computationResults,
          resultsWritingIndex, problemCount, degreeOfParallelism) -> int
  Verify(problems, problemsReadingIndex, problemCount, degreeOfParallelism) -> int
  GetBestParallelism() -> int

Both return the index of the first automaton whose shortest word is longer
than (n-1)^2 (a counterexample to Cerny's conjecture), else -1.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _native
from .problem import Problem, records_from_problems, RECORD_LSTRIDE


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def word_stride_for(max_n: int) -> int:
    return max(1, ((max(max_n, 2) - 1) ** 2 + 63) // 64)


class Engine:
    """One native handle: streams, device buffers, kernel plan."""

    def __init__(self, device: int = -1, slack: int = 0, autotune: bool = False, use_graph: bool = False,
                 slots_per_warp: int = 0, warps_per_cta: int = 0, queue_smem: int = 0, chunk: int = 0,
                 small_kernel: int = 0, lane_ring: int = 0, lane_refill: int = 0, lane_warps: int = 0,
                 lane_tail: int = 0, streams: int = 0,
                 level_arena_bytes: int = 0, tune_cache: Optional[str] = None, wait_polls: int = 0):
        self.lib = _native.load()
        cfg = _native.Config()
        self.lib.sbfs_config_default(ctypes.byref(cfg))
        cfg.device = device
        cfg.slack = slack
        cfg.autotune = int(autotune)
        cfg.use_graph = int(use_graph)
        cfg.slots_per_warp = slots_per_warp
        cfg.warps_per_cta = warps_per_cta
        cfg.queue_smem = queue_smem
        cfg.chunk = chunk
        cfg.small_kernel = small_kernel
        cfg.lane_ring = lane_ring
        cfg.lane_refill = lane_refill
        cfg.lane_tail = lane_tail
        cfg.lane_warps = lane_warps
        cfg.streams = streams
        cfg.level_arena_bytes = level_arena_bytes
        self._tune_cache = tune_cache.encode() if tune_cache else None
        cfg.tune_cache = self._tune_cache
        cfg.wait_polls = wait_polls
        h = ctypes.c_void_p()
        st = self.lib.sbfs_create(ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            msg = self.lib.sbfs_last_error(None)
            raise _native.SbfsError(st, msg.decode() if msg else "")
        self.handle = h
        self.last_stats: Optional[dict] = None

    def close(self):
        if getattr(self, "handle", None):
            self.lib.sbfs_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def plan(self) -> dict:
        """Kernel and shape per size class, as the native plan describes it."""
        import json
        need = self.lib.sbfs_describe_plan(self.handle, None, 0)
        buf = ctypes.create_string_buffer(max(need, 1))
        self.lib.sbfs_describe_plan(self.handle, buf, len(buf))
        return json.loads(buf.value.decode()) if buf.value else {}

    def best_parallelism(self) -> int:
        return int(self.lib.sbfs_best_parallelism(self.handle))

    def _prep(self, recs, ns, n, lstride):
        recs = np.ascontiguousarray(recs, dtype=np.uint8)
        if recs.ndim != 2 or recs.shape[1] != 2 * lstride:
            raise ValueError(f"records must have shape (count, {2 * lstride})")
        ns_arr = None if ns is None else np.ascontiguousarray(ns, dtype=np.uint8)
        if ns_arr is not None and ns_arr.shape[0] != recs.shape[0]:
            raise ValueError("ns must have one entry per record")
        max_n = int(ns_arr.max()) if (ns_arr is not None and ns_arr.size) else int(n)
        return recs, ns_arr, max_n

    def solve(self, recs, ns=None, n: int = 0, lstride: int = RECORD_LSTRIDE, words: bool = True,
              word_stride: Optional[int] = None, plain: bool = False, out=None):
        """Solve every automaton.  Returns dict(len, words, word_stride,
        first_violation, stats).  ``out`` may pass preallocated (len, words)."""
        recs, ns_arr, max_n = self._prep(recs, ns, n, lstride)
        count = recs.shape[0]
        ws = int(word_stride or word_stride_for(max_n))
        if out is not None:
            out_len, out_words = out
        else:
            out_len = np.empty(count, dtype=np.int32)
            out_words = np.empty((count, ws), dtype=np.uint64) if words else None
        fv = ctypes.c_int64(-1)
        stats = _native.Stats()
        fn = self.lib.sbfs_solve_plain if plain else self.lib.sbfs_solve_batch
        st = fn(self.handle, _ptr(recs), lstride, _ptr(ns_arr), int(n), count, _ptr(out_len),
                _ptr(out_words) if words else None, ws if words else 0, ctypes.byref(fv),
                ctypes.byref(stats))
        self.last_stats = stats.as_dict()
        _native.check(self.handle, st)
        return {"len": out_len, "words": out_words if words else None, "word_stride": ws,
                "first_violation": fv.value, "stats": self.last_stats}

    def solve_device(self, d_maps, lstride: int, count: int, n: int = 0, d_ns=None, max_n: int = 0,
                     d_len=None, d_words=None, word_stride: int = 0, d_first_violation=None,
                     stream=None):
        """Enqueue a solve on device buffers (torch tensors or raw device
        addresses); returns immediately.  Call ``wait_device`` for status."""
        def addr(x):
            if x is None:
                return None
            return ctypes.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else int(x))
        st_ptr = None
        if stream is not None:
            st_ptr = ctypes.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))
        st = self.lib.sbfs_solve_batch_device(self.handle, addr(d_maps), lstride, addr(d_ns), int(n),
                                              int(max_n), int(count), addr(d_len), addr(d_words),
                                              int(word_stride), addr(d_first_violation), st_ptr)
        _native.check(self.handle, st)

    def wait_device(self) -> dict:
        stats = _native.Stats()
        st = self.lib.sbfs_device_wait(self.handle, ctypes.byref(stats))
        self.last_stats = stats.as_dict()
        _native.check(self.handle, st)
        return self.last_stats

    def verify(self, recs, ns=None, n: int = 0, lstride: int = RECORD_LSTRIDE, lengths: bool = True):
        """Lengths only (IComputable.Verify); returns dict(len, first_violation, stats)."""
        recs, ns_arr, _ = self._prep(recs, ns, n, lstride)
        count = recs.shape[0]
        out_len = np.empty(count, dtype=np.int32) if lengths else None
        fv = ctypes.c_int64(-1)
        stats = _native.Stats()
        st = self.lib.sbfs_verify_batch(self.handle, _ptr(recs), lstride, _ptr(ns_arr), int(n), count,
                                        _ptr(out_len), ctypes.byref(fv), ctypes.byref(stats))
        self.last_stats = stats.as_dict()
        _native.check(self.handle, st)
        return {"len": out_len, "first_violation": fv.value, "stats": self.last_stats}


@dataclass
class ComputationResult:
    """Mirror of GPGPU/Shared/ComputationResult.cs:9-20 (fields the path fills)."""

    isSynchronizable: bool = False
    shortestSynchronizingWord: Optional[List[bool]] = None
    shortestSynchronizingWordLength: int = 0
    size: int = 0
    algorithmName: str = ""
    computationType: str = "GPU"
    discoveredVertices: int = 0
    queueBreadth: int = 0


def word_bits_to_bools(bits: np.ndarray, length: int) -> List[bool]:
    """uint64 word bits -> the reference's bool[] (true = letter b, index 0 first)."""
    return [bool((int(bits[k >> 6]) >> (k & 63)) & 1) for k in range(length)]


class SlimGPUNative:
    """IComputable (GPGPU/Interfaces/IComputable.cs:11-20) on the B200 engine."""

    def __init__(self, engine: Optional[Engine] = None, **engine_kwargs):
        self.engine = engine or Engine(**engine_kwargs)

    def GetBestParallelism(self) -> int:  # IComputable.cs:19
        return self.engine.best_parallelism()

    def Compute(self, problemsToSolve: Sequence[Problem], problemsReadingIndex: int,
                computationResults: Optional[list], resultsWritingIndex: int, problemCount: int,
                degreeOfParallelism: int) -> int:  # IComputable.cs:14
        if problemCount == 0:
            return -1
        probs = problemsToSolve[problemsReadingIndex:problemsReadingIndex + problemCount]
        recs, ns = records_from_problems(probs)
        if computationResults is None:
            r = self.engine.verify(recs, ns=ns, lengths=False)
            fv = r["first_violation"]
            return -1 if fv < 0 else problemsReadingIndex + fv
        r = self.engine.solve(recs, ns=ns, words=True)
        for i, p in enumerate(probs):
            L = int(r["len"][i])
            res = ComputationResult(size=p.size, algorithmName=type(self).__name__)
            if L >= 0:
                res.isSynchronizable = True
                res.shortestSynchronizingWordLength = L
                res.shortestSynchronizingWord = word_bits_to_bools(r["words"][i], L)
            computationResults[resultsWritingIndex + i] = res
        fv = r["first_violation"]
        return -1 if fv < 0 else resultsWritingIndex + fv

    def Verify(self, problemsToSolve: Sequence[Problem], problemsReadingIndex: int, problemCount: int,
               degreeOfParallelism: int) -> int:  # IComputable.cs:17
        return self.Compute(problemsToSolve, problemsReadingIndex, None, -1, problemCount,
                            degreeOfParallelism)


CERNY_FAILED_CSV = "./cernyFailed.csv"


def verify_and_report(solver, problems: Sequence[Problem], path: str = CERNY_FAILED_CSV) -> int:
    """The benchmark's Verify step (GPGPU/Program.cs:108-129): run
    ``solver.Verify`` over all ``problems`` at its best parallelism; when an
    automaton's shortest word is longer than (n-1)^2, append that automaton's
    ``ToString()`` to ``path`` (``File.AppendAllText``: no separator, as the
    reference writes it) and return its index, else return -1."""
    result = solver.Verify(problems, 0, len(problems), solver.GetBestParallelism())
    if result >= 0:
        with open(path, "a", encoding="utf-8") as f:
            f.write(str(problems[result]))
    return result


def read_cerny_failed(path: str = CERNY_FAILED_CSV) -> List[Problem]:
    """Automata appended by :func:`verify_and_report` (or by the reference),
    split at the ``]][[`` joints the separator-less appends leave."""
    with open(path, encoding="utf-8") as f:
        text = f.read().strip()
    if not text:
        return []
    parts = text.replace("]][[", "]]\n[[").split("\n")
    return [Problem.parse(p) for p in parts if p.strip()]

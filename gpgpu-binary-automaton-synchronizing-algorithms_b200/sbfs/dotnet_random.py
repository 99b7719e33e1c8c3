""".NET ``System.Random`` and the reference's seeded input batches.

The reference draws every random automaton with .NET Framework's
``System.Random`` (``SharedDefinitions/Problem.cs:32-58``):

  FillArrayOfProblems(problems, count, n, seed):
      master = Random(seed)
      problems[i] = GenerateProblem(n, master.Next())     for i in 0..count-1
  GenerateProblem(n, seed):
      r = Random(seed)
      A[i] = r.Next(0, n); B[i] = r.Next(0, n)            for i in 0..n-1

and the GPGPU benchmark fills ``count`` automata with seed ``1234567 + count``
(``GPGPU/Program.cs:58,94``); the correctness test uses seeds 12456..12465 at
n = 13 (``AlgorithmCorrectnessTestProject/IntegrityTest.cs:71-79``).

``System.Random`` is Knuth's subtractive generator (a 55-entry table filled
from the seed by the additive recurrence at stride 21 and stirred four times;
outputs are differences at lags 55 and 34, taken modulo 2^31 - 1).
``DotnetRandom`` restates it in Python for single automata and small
cross-checks; ``fill_array_of_problems`` runs the same generator in the native
library (``sbfs_generate_reference_batch``), which is what batches of millions
need.
"""
from __future__ import annotations

from typing import List

import numpy as np

from . import _native
from .problem import Problem, RECORD_LSTRIDE

_MBIG = 2147483647
_MSEED = 161803398


def _wrap32(v: int) -> int:
    """C# unchecked int arithmetic: wrap to the signed 32-bit range.  Seeds
    above 161803398 make the table's first entry negative and the stirring
    loop overflows, so the wrap is part of the generator."""
    return ((v + (1 << 31)) & 0xFFFFFFFF) - (1 << 31)

#: seed base of the GPGPU benchmark batches (GPGPU/Program.cs:58)
BENCHMARK_SEED = 1234567


class DotnetRandom:
    """``System.Random(seed)`` of .NET Framework: ``Next()``, ``Next(max)``,
    ``Next(min, max)`` and ``NextDouble()``."""

    def __init__(self, seed: int):
        seed = int(seed)
        if not -(1 << 31) <= seed < (1 << 31):
            raise ValueError("seed must be a 32-bit signed integer")
        sub = _MBIG if seed == -(1 << 31) else abs(seed)
        t = [0] * 56
        mj = _MSEED - sub
        t[55] = mj
        mk = 1
        for i in range(1, 55):
            ii = (21 * i) % 55
            t[ii] = mk
            mk = _wrap32(mj - mk)
            if mk < 0:
                mk += _MBIG
            mj = t[ii]
        for _ in range(4):
            for i in range(1, 56):
                t[i] = _wrap32(t[i] - t[1 + (i + 30) % 55])
                if t[i] < 0:
                    t[i] += _MBIG
        self._t = t
        self._next = 0
        self._nextp = 21

    def _sample_int(self) -> int:
        self._next = 1 if self._next + 1 >= 56 else self._next + 1
        self._nextp = 1 if self._nextp + 1 >= 56 else self._nextp + 1
        r = _wrap32(self._t[self._next] - self._t[self._nextp])
        if r == _MBIG:
            r -= 1
        if r < 0:
            r += _MBIG
        self._t[self._next] = r
        return r

    def NextDouble(self) -> float:
        return self._sample_int() * (1.0 / _MBIG)

    def Next(self, a: int = None, b: int = None) -> int:
        if a is None:
            return self._sample_int()
        lo, hi = (0, a) if b is None else (a, b)
        if lo > hi or (b is None and hi < 0):
            raise ValueError("minValue > maxValue")
        rng = hi - lo
        if rng > _MBIG:
            raise ValueError("ranges wider than 2^31 - 1 are not restated")
        return int(self.NextDouble() * rng) + lo


def generate_problem(n: int, seed: int) -> Problem:
    """``Problem.GenerateProblem`` (Problem.cs:41-58)."""
    r = DotnetRandom(seed)
    a: List[int] = []
    b: List[int] = []
    for _ in range(n):
        a.append(r.Next(0, n))
        b.append(r.Next(0, n))
    return Problem(a, b, n)


def fill_array_of_problems_py(count: int, n: int, seed: int) -> List[Problem]:
    """``Problem.FillArrayOfProblems`` (Problem.cs:32-39) in Python (small counts)."""
    master = DotnetRandom(seed)
    return [generate_problem(n, master.Next()) for _ in range(count)]


def fill_array_of_problems(count: int, n: int, seed: int, lstride: int = RECORD_LSTRIDE) -> np.ndarray:
    """``Problem.FillArrayOfProblems`` as packed records (``2 * lstride`` bytes
    each, ``a = rec[:n]``, ``b = rec[lstride:lstride + n]``), generated by the
    native library."""
    count, n, lstride = int(count), int(n), int(lstride)
    out = np.empty((count, 2 * lstride), dtype=np.uint8)
    lib = _native.load()
    st = lib.sbfs_generate_reference_batch(count, n, int(seed), out.ctypes.data if count else None, lstride)
    if st != 0:
        raise _native.SbfsError(st, f"sbfs_generate_reference_batch(count={count}, n={n}, lstride={lstride})")
    return out


def benchmark_batch(count: int, n: int, lstride: int = RECORD_LSTRIDE) -> np.ndarray:
    """The batch GPGPU/Program.cs:94 solves for ``count`` automata of ``n`` states."""
    return fill_array_of_problems(count, n, BENCHMARK_SEED + int(count), lstride)


def random_next(seed: int, count: int) -> np.ndarray:
    """The first ``count`` values of ``new Random(seed).Next()`` (native)."""
    out = np.empty(int(count), dtype=np.int32)
    lib = _native.load()
    st = lib.sbfs_dotnet_random_next(int(seed), int(count), out.ctypes.data if count else None)
    if st != 0:
        raise _native.SbfsError(st, f"sbfs_dotnet_random_next(count={count})")
    return out

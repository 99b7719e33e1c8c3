"""Automaton inputs: the reference's ``Problem`` type, its generators and the
packed record layout the native library reads.

Reference: ``SharedDefinitions/Problem.cs``.
  * ``Problem`` (:7-11) -- two transition maps ``stateTransitioningMatrixA/B``
    of length ``size``.
  * ``GenerateWorstCase`` (:13-29) -- the Cerny automaton C_n: A sends 0 to 1 and
    fixes every other state, B is the cycle i -> i+1 mod n.  Its shortest
    synchronizing word has length exactly (n-1)^2.
  * ``FillArrayOfProblems`` / ``GenerateProblem`` (:32-58) -- uniform random maps.
    The reference draws them from .NET ``System.Random``; here a counter-based
    splitmix64 stream gives reproducible, vectorisable inputs instead (the .NET
    generator itself is in :mod:`sbfs.dotnet_random`).

Record layout: automaton i is ``2 * lstride`` bytes; ``a[j] = rec[j]`` and
``b[j] = rec[lstride + j]`` for j < n.  ``lstride = 32`` is the general 64-byte
record (any n <= 28, mixed sizes); ``lstride = n`` packs a uniform batch
tightly (24 bytes per automaton at n = 12).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Iterable, List, Optional, Sequence

import numpy as np

MAX_N = 28
RECORD_LSTRIDE = 32

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


@dataclass
class Problem:
    """Mirror of ``SharedDefinitions/Problem.cs:7-11``."""

    stateTransitioningMatrixA: List[int]
    stateTransitioningMatrixB: List[int]
    size: int = field(default=-1)

    def __post_init__(self):
        if self.size < 0:
            self.size = len(self.stateTransitioningMatrixA)

    def __str__(self) -> str:  # Problem.cs:60-79, "[[a...],[b...]]"
        a = ",".join(str(int(v)) for v in self.stateTransitioningMatrixA[: self.size])
        b = ",".join(str(int(v)) for v in self.stateTransitioningMatrixB[: self.size])
        return f"[[{a}],[{b}]]"

    @staticmethod
    def parse(text: str) -> "Problem":
        """Inverse of ``__str__`` (the ``cernyFailed.csv`` line format)."""
        body = text.strip()
        if not (body.startswith("[[") and body.endswith("]]")):
            raise ValueError(f"not a [[a..],[b..]] automaton: {text!r}")
        left, right = body[2:-2].split("],[")
        a = [int(v) for v in left.split(",")]
        b = [int(v) for v in right.split(",")]
        if len(a) != len(b):
            raise ValueError("letters a and b have different lengths")
        return Problem(a, b, len(a))


def generate_worst_case(n: int) -> Problem:
    """``Problem.GenerateWorstCase`` (Problem.cs:13-29): C_n with the reference's
    letter names (A merges 0 into 1, B is the cycle)."""
    if n < 3:
        raise ValueError("wrong number!")  # Problem.cs:15-16
    a = [1 if i == 0 else i for i in range(n)]
    b = [0 if i + 1 == n else i + 1 for i in range(n)]
    return Problem(a, b, n)


# ---------------------------------------------------------------------------
# counter-based generator: value(seed, counter) = splitmix64(splitmix64(seed) + counter)
# ---------------------------------------------------------------------------

def _splitmix64(x: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
        return z ^ (z >> np.uint64(31))


def hash_stream(seed: int, counters: np.ndarray) -> np.ndarray:
    """64-bit hashes for the given counters under ``seed``."""
    base = _splitmix64(np.array([seed & 0xFFFFFFFFFFFFFFFF], dtype=np.uint64))[0]
    with np.errstate(over="ignore"):
        return _splitmix64((counters.astype(np.uint64) + base) & _M64)


def _below(h: np.ndarray, bound) -> np.ndarray:
    """Multiply-shift range reduction of the high 32 bits into [0, bound)."""
    hi = h >> np.uint64(32)
    return ((hi * np.asarray(bound, dtype=np.uint64)) >> np.uint64(32)).astype(np.int64)


def uniform_maps(count: int, n, seed: int, lstride: int = RECORD_LSTRIDE) -> np.ndarray:
    """``count`` automata with independent uniform maps [n] -> [n] for a and b.

    ``n`` is an int or a per-automaton array.  Returns uint8 records of shape
    ``(count, 2 * lstride)``; bytes past n are zero.
    """
    ns = np.broadcast_to(np.asarray(n, dtype=np.int64), (count,))
    if count and (ns.max() > lstride or ns.min() < 1):
        raise ValueError("n out of range for the record stride")
    idx = np.arange(count, dtype=np.uint64)[:, None] * np.uint64(64)
    cols = np.arange(2 * lstride, dtype=np.uint64)[None, :]
    letter = cols // np.uint64(lstride)
    state = cols % np.uint64(lstride)
    ctr = idx + letter * np.uint64(32) + state
    vals = _below(hash_stream(seed, ctr), ns[:, None])
    valid = state.astype(np.int64) < ns[:, None]
    return np.where(valid, vals, 0).astype(np.uint8)


def uniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """n drawn uniformly from lo..hi (inclusive)."""
    h = hash_stream(seed ^ 0x5A5A5A5A, np.arange(count, dtype=np.uint64))
    return (lo + _below(h, hi - lo + 1)).astype(np.uint8)


def log_uniform_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """n log-uniform over lo..hi (inclusive), rounded down."""
    h = hash_stream(seed ^ 0x3C3C3C3C, np.arange(count, dtype=np.uint64))
    u = (h >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    v = np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))
    return np.clip(np.floor(v), lo, hi).astype(np.uint8)


def cerny_record(n: int, lstride: int = RECORD_LSTRIDE) -> np.ndarray:
    """C_n with the letter names used by the benchmark configurations:
    a is the cycle i -> i+1 mod n, b sends 0 to 1 and fixes the rest.  (The
    reference's ``GenerateWorstCase`` swaps the names; the length is the same.)"""
    rec = np.zeros(2 * lstride, dtype=np.uint8)
    rec[:n] = [(i + 1) % n for i in range(n)]
    rec[lstride:lstride + n] = [1 if i == 0 else i for i in range(n)]
    return rec


def perm_merge_record(n: int, seed: int, lstride: int = RECORD_LSTRIDE) -> np.ndarray:
    """Slowly-synchronising family: a is a uniform random permutation, b is the
    identity except that one random pair (p, q) is merged (b[p] = q)."""
    h = hash_stream(seed, np.arange(n + 2, dtype=np.uint64))
    perm = list(range(n))
    for i in range(n - 1, 0, -1):  # Fisher-Yates
        j = int(_below(h[i:i + 1], i + 1)[0])
        perm[i], perm[j] = perm[j], perm[i]
    p = int(_below(h[n:n + 1], n)[0])
    q = int(_below(h[n + 1:n + 2], n - 1)[0])
    if q >= p:
        q += 1
    rec = np.zeros(2 * lstride, dtype=np.uint8)
    rec[:n] = perm
    b = list(range(n))
    b[p] = q
    rec[lstride:lstride + n] = b
    return rec


def records_from_problems(problems: Sequence[Problem], lstride: int = RECORD_LSTRIDE):
    """Pack ``Problem`` objects into records plus a per-automaton n array."""
    recs = np.zeros((len(problems), 2 * lstride), dtype=np.uint8)
    ns = np.zeros(len(problems), dtype=np.uint8)
    for i, p in enumerate(problems):
        n = int(p.size)
        if not 1 <= n <= min(lstride, MAX_N):
            raise ValueError(f"problem {i}: size {n} out of range")
        recs[i, :n] = p.stateTransitioningMatrixA[:n]
        recs[i, lstride:lstride + n] = p.stateTransitioningMatrixB[:n]
        ns[i] = n
    return recs, ns


def problems_from_records(recs: np.ndarray, ns, lstride: int = RECORD_LSTRIDE) -> List[Problem]:
    ns = np.broadcast_to(np.asarray(ns), (recs.shape[0],))
    out = []
    for i in range(recs.shape[0]):
        n = int(ns[i])
        out.append(Problem(recs[i, :n].tolist(), recs[i, lstride:lstride + n].tolist(), n))
    return out


def repack(recs: np.ndarray, lstride_from: int, lstride_to: int) -> np.ndarray:
    """Change the record stride (e.g. 64-byte records -> tight 2n-byte records)."""
    out = np.zeros((recs.shape[0], 2 * lstride_to), dtype=np.uint8)
    k = min(lstride_from, lstride_to)
    out[:, :k] = recs[:, :k]
    out[:, lstride_to:lstride_to + k] = recs[:, lstride_from:lstride_from + k]
    return out

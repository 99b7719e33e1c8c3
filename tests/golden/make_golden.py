"""Generates tests/golden/small_automata.npz: seeded small automata with their
shortest synchronizing word lengths found WITHOUT power-set BFS, so the fixtures
pin the oracle independently of its own algorithm:

  * synchronizing or not: the pair criterion -- an automaton synchronizes iff
    every pair of states can be merged by some word (fixpoint over pairs);
  * length: breadth-first enumeration of all words (no visited set, no
    deduplication of subsets): the smallest L such that some word of length L
    maps the full state set to a single state.

Also records the reference's known answers (AlgorithmCorrectnessTestProject/
SimpleAutomataTests.cs:14-35): Problem.GenerateWorstCase(n) has length (n-1)^2.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "gpgpu-binary-automaton-synchronizing-algorithms_b200"))
from sbfs import problem as P  # noqa: E402

LSTRIDE = 32


def pair_synchronizing(a, b, n):
    merge = np.zeros((n, n), dtype=bool)
    np.fill_diagonal(merge, True)
    changed = True
    while changed:
        changed = False
        for p in range(n):
            for q in range(n):
                if not merge[p, q] and (merge[a[p], a[q]] or merge[b[p], b[q]]):
                    merge[p, q] = True
                    changed = True
    return bool(merge.all())


def word_search_length(a, b, n, cap=22):
    """Smallest L with a word of length L collapsing all states, by enumerating
    words level by level (2^L sets at level L, no deduplication)."""
    a = np.asarray(a, dtype=np.int64)
    b = np.asarray(b, dtype=np.int64)
    sets = np.array([(1 << n) - 1], dtype=np.int64)
    sa = (1 << a).astype(np.int64)
    sb = (1 << b).astype(np.int64)

    def image(s, single):
        out = np.zeros_like(s)
        for j in range(n):
            out |= np.where((s >> j) & 1, single[j], 0)
        return out

    for L in range(1, cap + 1):
        sets = np.concatenate([image(sets, sa), image(sets, sb)])
        if np.any((sets & (sets - 1)) == 0):
            return L
        sets = np.unique(sets) if sets.size > (1 << 16) else sets  # bound memory only
    return None


def main():
    rows, ns, lens = [], [], []
    rng_seed = 0x5EED
    # exhaustive n = 2 (16 automata) and n = 3 (729 automata)
    for n in (2, 3):
        m = n ** n
        for ia in range(m):
            for ib in range(m):
                a = [(ia // n ** j) % n for j in range(n)]
                b = [(ib // n ** j) % n for j in range(n)]
                rows.append((a, b)); ns.append(n)
    # seeded random n = 4..6
    for n, cnt in ((4, 400), (5, 300), (6, 150)):
        recs = P.uniform_maps(cnt, n, rng_seed + n)
        for r in recs:
            rows.append((list(r[:n]), list(r[LSTRIDE:LSTRIDE + n]))); ns.append(n)
    recs = np.zeros((len(rows), 2 * LSTRIDE), dtype=np.uint8)
    for i, (a, b) in enumerate(rows):
        n = ns[i]
        recs[i, :n] = a
        recs[i, LSTRIDE:LSTRIDE + n] = b
        sync = pair_synchronizing(a, b, n)
        L = word_search_length(a, b, n) if sync else None
        if sync and L is None:
            raise RuntimeError("word search cap too small")
        lens.append(L if sync else -1)
    ns = np.array(ns, dtype=np.uint8)
    lens = np.array(lens, dtype=np.int32)
    cerny_n = np.arange(3, 29, dtype=np.int32)
    cerny_len = (cerny_n - 1) ** 2
    np.savez_compressed(os.path.join(HERE, "small_automata.npz"), recs=recs, ns=ns, lens=lens,
                        cerny_n=cerny_n, cerny_len=cerny_len)
    print(f"{len(lens)} automata, {int((lens < 0).sum())} non-synchronizing, max length {lens.max()}")


if __name__ == "__main__":
    main()

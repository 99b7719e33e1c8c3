"""Pins the CPU oracle (oracle/sbfs_oracle.c) before it is trusted as the checker.

* the reference's known answers: Problem.GenerateWorstCase(n) has shortest
  word length (n-1)^2 (AlgorithmCorrectnessTestProject/SimpleAutomataTests.cs:14-35,
  IntegrityTest.cs:44-62), extended from n <= 13 to n <= 20;
* golden fixtures from an independent word enumeration (tests/golden/make_golden.py),
  exhaustive for n = 2, 3 and seeded for n = 4..6;
* the two reference CPU variants agree (SlimCPUUntweaked vs SlimCPU4bits13);
* every word replays to a singleton (Verify.cs:12-54).
"""
import os

import numpy as np
import pytest

from sbfs import problem as P

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "small_automata.npz")


def test_worst_case_reference_letters(oracle_mod):
    # Problem.GenerateWorstCase as the reference builds it (A merges, B cycles)
    for n in range(3, 14):
        p = P.generate_worst_case(n)
        recs, ns = P.records_from_problems([p])
        r = oracle_mod.solve(recs, ns=ns)
        assert r["len"][0] == (n - 1) ** 2
        bad, _ = oracle_mod.replay(recs, r["len"], r["words"], ns=ns)
        assert bad == 0


@pytest.mark.parametrize("n", list(range(3, 21)))
def test_cerny_family_benchmark_letters(oracle_mod, n):
    rec = P.cerny_record(n)[None, :]
    r = oracle_mod.solve(rec, n=n)
    assert r["len"][0] == (n - 1) ** 2
    bad, _ = oracle_mod.replay(rec, r["len"], r["words"], n=n)
    assert bad == 0


def test_golden_fixtures(oracle_mod):
    g = np.load(GOLDEN)
    r = oracle_mod.solve(g["recs"], ns=g["ns"], threads=2)
    np.testing.assert_array_equal(r["len"], g["lens"])
    bad, _ = oracle_mod.replay(g["recs"], r["len"], r["words"], ns=g["ns"])
    assert bad == 0


def test_golden_has_both_outcomes():
    g = np.load(GOLDEN)
    assert (g["lens"] < 0).sum() > 0 and (g["lens"] > 0).sum() > 0
    assert (g["cerny_len"] == (g["cerny_n"] - 1) ** 2).all()


@pytest.mark.parametrize("n", [4, 8, 12])
def test_nibble_variant_matches_untweaked(oracle_mod, n):
    recs = P.uniform_maps(3000, n, 7 + n)
    a = oracle_mod.solve(recs, n=n, words=False, threads=3)
    tight = P.repack(recs, 32, n)
    b = oracle_mod.verify4(tight, n=n, lstride=n, write_len=True, threads=2)
    np.testing.assert_array_equal(a["len"], b["len"])
    assert a["expanded"] == b["expanded"]


def test_threads_do_not_change_results(oracle_mod):
    recs = P.uniform_maps(5000, 10, 99)
    a = oracle_mod.solve(recs, n=10, threads=1)
    b = oracle_mod.solve(recs, n=10, threads=7)
    np.testing.assert_array_equal(a["len"], b["len"])
    np.testing.assert_array_equal(a["words"], b["words"])


def test_mixed_sizes_and_large_n(oracle_mod):
    ns = P.uniform_sizes(400, 6, 22, 3)
    recs = P.uniform_maps(400, ns, 4)
    r = oracle_mod.solve(recs, ns=ns, threads=4)
    bad, _ = oracle_mod.replay(recs, r["len"], r["words"], ns=ns)
    assert bad == 0
    # each automaton alone gives the same answer
    for i in range(0, 400, 37):
        one = oracle_mod.solve(recs[i:i + 1], ns=ns[i:i + 1])
        assert one["len"][0] == r["len"][i]


def test_n1_matches_reference_behaviour(oracle_mod):
    # SlimCPUUntweaked marks the full set visited before expanding it, so an
    # automaton with one state never generates an undiscovered singleton.
    rec = np.zeros((1, 64), dtype=np.uint8)
    assert oracle_mod.solve(rec, n=1)["len"][0] == -1


def test_violation_reporting_with_slack(oracle_mod):
    # C_5 has length 16 = (5-1)^2; lowering the bound by 1 makes it a violation
    recs = np.stack([P.uniform_maps(1, 5, 1)[0], P.cerny_record(5), P.cerny_record(5)])
    assert oracle_mod.solve(recs, n=5)["first_violation"] == -1
    assert oracle_mod.solve(recs, n=5, slack=1)["first_violation"] == 1


def test_replay_detects_a_planted_bad_word(oracle_mod):
    recs = P.uniform_maps(200, 7, 5)
    r = oracle_mod.solve(recs, n=7)
    i = int(np.argmax(r["len"] > 2))
    words = r["words"].copy()
    words[i, 0] ^= 1  # flip the first letter of one word
    bad, ok = oracle_mod.replay(recs, r["len"], words, n=7)
    # flipping a letter can still synchronize by luck; the length check stays
    assert bad in (0, 1) and ok[i] in (2, 3)
    lens = r["len"].copy()
    lens[i] = 100  # beyond (n-1)^2 and beyond the stored word
    bad, ok = oracle_mod.replay(recs, lens, r["words"], n=7)
    assert bad == 1 and ok[i] == 0


def test_invalid_records_rejected(oracle_mod):
    rec = np.zeros((1, 64), dtype=np.uint8)
    rec[0, 3] = 9  # state 9 with n = 5
    with pytest.raises(ValueError):
        oracle_mod.solve(rec, n=5)


@pytest.mark.parametrize("n", [6, 10, 14, 18])
def test_two_closed_components_never_synchronize(oracle_mod, n):
    """States 0..h-1 and h..n-1 each closed under both letters: no word maps a
    state of one half into the other, so no word synchronizes, however the
    halves behave alone.  Each half alone is a random automaton; the oracle
    must report -1 for the union (the GPU hand-off test plants these)."""
    h = n // 2
    rows = []
    for seed in range(5):
        lo = P.uniform_maps(1, h, 300 + seed)[0]
        hi = P.uniform_maps(1, n - h, 400 + seed)[0]
        rec = np.zeros(64, dtype=np.uint8)
        for letter in range(2):
            base = 32 * letter
            rec[base:base + h] = lo[base:base + h]
            rec[base + h:base + n] = hi[base:base + n - h] + h
        rows.append(rec)
    recs = np.stack(rows)
    assert (oracle_mod.solve(recs, n=n, words=False)["len"] == -1).all()


def test_permutation_automata_never_synchronize(oracle_mod):
    """Both letters permutations: every image of the full set is the full set."""
    rng = np.random.default_rng(11)
    recs = np.zeros((20, 64), dtype=np.uint8)
    ns = rng.integers(2, 21, 20).astype(np.uint8)
    for i, n in enumerate(ns):
        recs[i, :n] = rng.permutation(int(n))
        recs[i, 32:32 + n] = rng.permutation(int(n))
    assert (oracle_mod.solve(recs, ns=ns, words=False)["len"] == -1).all()

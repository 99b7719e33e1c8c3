""".NET System.Random restatement and the reference's seeded batches (CPU).

* known answers: the first outputs of ``new Random(seed).Next()`` on .NET
  Framework for seeds 0, 1 and 42, as published for that runtime;
* the native generator (sbfs_generate_reference_batch / sbfs_dotnet_random_next)
  and the Python restatement agree on every seed class, including seeds above
  161803398 where C#'s unchecked int arithmetic wraps while the table is stirred;
* Problem.FillArrayOfProblems (SharedDefinitions/Problem.cs:32-58) layout: A
  then B per state, values in [0, n), padding bytes zero;
* GPGPU/Program.cs:94's benchmark seed 1234567 + count;
* the oracle on an IntegrityTest batch (AlgorithmCorrectnessTestProject/
  IntegrityTest.cs:71-79: n = 13, seeds from 12456): Cerny's bound holds and
  every word replays.
"""
import numpy as np
import pytest

import sbfs
from sbfs import dotnet_random as D

# new Random(seed).Next() x 5 on .NET Framework (published outputs of the runtime)
KNOWN = {
    0: [1559595546, 1755192844, 1649316166, 1198642031, 442452829],
    1: [534011718, 237820880, 1002897798, 1657007234, 1412011072],
    42: [1434747710, 302596119, 269548474, 1122627734, 361709742],
}

SEEDS = [0, 1, 7, 42, 12456, 1234567, 161803397, 161803398, 161803399, 1959380556, (1 << 31) - 1,
         -1, -42, -161803399, -(1 << 31)]


@pytest.mark.parametrize("seed", sorted(KNOWN))
def test_known_answers(seed):
    r = D.DotnetRandom(seed)
    assert [r.Next() for _ in range(5)] == KNOWN[seed]
    assert D.random_next(seed, 5).tolist() == KNOWN[seed]


@pytest.mark.parametrize("seed", SEEDS)
def test_native_equals_restatement(seed):
    r = D.DotnetRandom(seed)
    py = [r.Next() for _ in range(300)]   # more than one pass over the 55-entry table
    assert D.random_next(seed, 300).tolist() == py
    assert all(0 <= v < 2147483647 for v in py)


def test_next_ranges():
    r = D.DotnetRandom(99)
    vals = [r.Next(0, 13) for _ in range(2000)]
    assert min(vals) == 0 and max(vals) == 12
    r = D.DotnetRandom(99)
    assert [r.Next(13) for _ in range(50)] == vals[:50]
    r = D.DotnetRandom(5)
    assert all(-3 <= r.Next(-3, 4) < 4 for _ in range(500))
    with pytest.raises(ValueError):
        D.DotnetRandom(1).Next(5, 2)
    with pytest.raises(ValueError):
        D.DotnetRandom(1 << 31)


@pytest.mark.parametrize("n", [1, 3, 12, 13, 20, 28])
def test_fill_array_of_problems(n):
    seed = 12456
    recs = D.fill_array_of_problems(400, n, seed)
    probs = D.fill_array_of_problems_py(400, n, seed)
    assert recs.shape == (400, 64)
    for i, p in enumerate(probs):
        assert recs[i, :n].tolist() == p.stateTransitioningMatrixA
        assert recs[i, 32:32 + n].tolist() == p.stateTransitioningMatrixB
    assert recs[:, n:32].max(initial=0) == 0 and recs[:, 32 + n:].max(initial=0) == 0
    assert recs[:, :n].max() < n and recs[:, 32:32 + n].max() < n
    # tight records hold the same automata
    tight = D.fill_array_of_problems(400, n, seed, lstride=n)
    np.testing.assert_array_equal(sbfs.repack(recs, 32, n), tight)


def test_single_problem_is_the_batch_member():
    master = D.DotnetRandom(777)
    seeds = [master.Next() for _ in range(3)]
    batch = D.fill_array_of_problems_py(3, 9, 777)
    for s, p in zip(seeds, batch):
        q = D.generate_problem(9, s)
        assert str(q) == str(p)


def test_benchmark_batch_seed():
    count = 5000
    np.testing.assert_array_equal(D.benchmark_batch(count, 12, lstride=12),
                                  D.fill_array_of_problems(count, 12, 1234567 + count, lstride=12))
    # the same batch spread over host threads and made in one piece
    big = D.fill_array_of_problems(70_000, 12, 31)
    np.testing.assert_array_equal(big[:400], D.fill_array_of_problems(400, 12, 31))


def test_bad_arguments():
    with pytest.raises(sbfs.SbfsError) as ei:
        D.fill_array_of_problems(10, 29, 1)
    assert ei.value.status == 1
    with pytest.raises(sbfs.SbfsError):
        D.fill_array_of_problems(10, 12, 1, lstride=8)
    with pytest.raises(sbfs.SbfsError):
        D.fill_array_of_problems(10, 0, 1)
    assert D.fill_array_of_problems(0, 12, 1).shape == (0, 64)


def test_oracle_on_integrity_batch(oracle_mod):
    n = 13
    recs = D.fill_array_of_problems(8192, n, 12456)
    ref = oracle_mod.solve(recs, n=n, words=True, threads=4)
    assert ref["first_violation"] == -1
    assert ref["len"].max() <= (n - 1) ** 2
    sync = ref["len"] >= 0
    assert 0.5 < sync.mean() < 1.0   # random binary automata mostly synchronise
    assert oracle_mod.replay(recs, ref["len"], ref["words"], n=n)[0] == 0


@pytest.mark.parametrize("seed", SEEDS)
def test_oracle_generator_equals_restatement(seed, oracle_mod):
    """The oracle's own System.Random (used by the CPU baseline, which must not
    load the product library) gives the same outputs and batches."""
    r = D.DotnetRandom(seed)
    assert oracle_mod.dotnet_random_next(seed, 300).tolist() == [r.Next() for _ in range(300)]


@pytest.mark.parametrize("n,lstride", [(1, 1), (8, 8), (12, 12), (13, 32), (20, 20), (28, 32)])
def test_oracle_batch_equals_native_batch(n, lstride, oracle_mod):
    seed = 1234567 + 5000
    mine = oracle_mod.fill_array_of_problems(5000, n, seed, lstride, threads=3)
    np.testing.assert_array_equal(mine, D.fill_array_of_problems(5000, n, seed, lstride=lstride))
    probs = D.fill_array_of_problems_py(50, n, seed)
    for i, p in enumerate(probs):
        assert mine[i, :n].tolist() == p.stateTransitioningMatrixA
        assert mine[i, lstride:lstride + n].tolist() == p.stateTransitioningMatrixB

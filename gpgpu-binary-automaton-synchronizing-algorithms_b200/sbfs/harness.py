"""Benchmark driver in the shape of the reference's ``GPGPU/Program.cs``.

``Program.Main`` (GPGPU/Program.cs:24-229) times every solver's ``Verify``
over growing batches of uniform random automata and keeps a CSV of
problems per second:

  * problem size 12, solvers listed in ``theSolver`` (:25-36);
  * batch sizes from 2^21 while below 2^25, each the previous one times
    ``sizeIncrease`` rounded (:72-77; the reference ships with growth 1, which
    never ends, and the commented-out 2^(1/8));
  * each batch is ``Problem.FillArrayOfProblems(problems, n, 12, 1234567 + n)``
    (:58, :94) -- regenerated here bit for bit by :mod:`sbfs.dotnet_random`;
  * per solver: ``Verify(problems, 0, n, GetBestParallelism())`` timed by a
    stopwatch (:108-111, :136-141); a counterexample to Cerny's conjecture is
    appended to ``./cernyFailed.csv`` in ``Problem.ToString`` form and ends the
    run (:112-124); otherwise ``round(n / seconds)`` is appended to the row
    (:153) and ``./gpgpu.csv`` is rewritten (:219);
  * CSV: header ``problemsize,problemcount,<solver class names>`` (:63-67), one
    row ``<problem size>,<n>,<rate>...`` per batch (:89-90).

Solvers here work on packed records (``2 * lstride`` bytes per automaton,
:mod:`sbfs.problem`) so that batches of millions need no Python objects:
anything with ``name``, ``GetBestParallelism()`` and
``verify_records(recs, n, lstride) -> int`` fits.  :class:`EngineSolver`
puts the B200 engine (batched or plain form) behind that interface.
"""
from __future__ import annotations

import argparse
import math
import time
from typing import List, Optional, Sequence

import numpy as np

from . import dotnet_random
from .problem import problems_from_records
from .solver import CERNY_FAILED_CSV, Engine

GPGPU_CSV = "./gpgpu.csv"


class EngineSolver:
    """The engine's Verify (``sbfs_verify_batch``, or ``sbfs_solve_plain`` --
    one launch per automaton -- with ``plain=True``) on packed records."""

    def __init__(self, engine: Optional[Engine] = None, plain: bool = False, name: Optional[str] = None,
                 **engine_kwargs):
        self.engine = engine or Engine(**engine_kwargs)
        self.plain = plain
        self.name = name or ("SlimGPUNativePlain" if plain else "SlimGPUNative")

    def GetBestParallelism(self) -> int:
        return self.engine.best_parallelism()

    def verify_records(self, recs: np.ndarray, n: int, lstride: int) -> int:
        if self.plain:
            r = self.engine.solve(recs, n=n, lstride=lstride, words=False, plain=True)
        else:
            r = self.engine.verify(recs, n=n, lstride=lstride, lengths=False)
        return int(r["first_violation"])


def batch_sizes(initial: int = 1 << 21, maximal: int = 1 << 25, growth: float = 2 ** 0.125,
                rounds: Optional[int] = None) -> List[int]:
    """The loop of Program.cs:76: n, round(n * growth), ... while n < maximal."""
    if growth <= 1.0 and rounds is None:
        raise ValueError("a growth of 1 never ends; give rounds")
    sizes, x = [], float(initial)
    n = int(initial)
    while n < maximal and (rounds is None or len(sizes) < rounds):
        sizes.append(n)
        x *= growth
        n = int(round(x))
    return sizes


def run(solvers: Sequence, problem_size: int = 12, sizes: Sequence[int] = (), csv_path: str = GPGPU_CSV,
        failed_path: str = CERNY_FAILED_CSV, seed: int = dotnet_random.BENCHMARK_SEED, log=print) -> dict:
    """Program.Main's benchmark loop.  Returns dict(csv=<text>, failed=<index or None>,
    rates={(n, solver name): problems per second})."""
    lstride = problem_size
    lines = ["problemsize,problemcount" + "".join("," + s.name for s in solvers)]
    rates = {}
    recs = None
    for n in sizes:
        row = f"{problem_size},{n}"
        if recs is None or recs.shape[0] != n:
            recs = dotnet_random.fill_array_of_problems(n, problem_size, seed + n, lstride=lstride)
        for s in solvers:
            t0 = time.perf_counter()
            result = s.verify_records(recs, problem_size, lstride)
            elapsed = time.perf_counter() - t0
            if result >= 0:
                bad = problems_from_records(recs[result:result + 1], problem_size, lstride)[0]
                with open(failed_path, "a", encoding="utf-8") as f:
                    f.write(str(bad))
                log(f"Cerny Conjecture is false.\nProblem description: {bad}")
                lines.append(row)
                with open(csv_path, "w", encoding="utf-8") as f:
                    f.write("\n".join(lines))
                return {"csv": "\n".join(lines), "failed": result, "rates": rates}
            rate = n / elapsed if elapsed > 0 else math.inf
            rates[(n, s.name)] = rate
            row += f",{round(rate)}"
            log(f"{s.name} using {s.GetBestParallelism()} parallelism in {elapsed * 1e3:.2f}ms. "
                f"Problems per second: {rate:.2f}. Time per problem {elapsed * 1e3 / n}ms")
        lines.append(row)
        with open(csv_path, "w", encoding="utf-8") as f:
            f.write("\n".join(lines))
    return {"csv": "\n".join(lines), "failed": None, "rates": rates}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Program.cs-style benchmark: Verify rates over growing batches")
    ap.add_argument("--problem-size", type=int, default=12)
    ap.add_argument("--initial", type=int, default=1 << 21)
    ap.add_argument("--maximal", type=int, default=1 << 25)
    ap.add_argument("--growth", type=float, default=2 ** 0.125)
    ap.add_argument("--rounds", type=int, default=None)
    ap.add_argument("--plain", action="store_true", help="also time the plain form (one launch per automaton)")
    ap.add_argument("--csv", default=GPGPU_CSV)
    ap.add_argument("--failed", default=CERNY_FAILED_CSV)
    ap.add_argument("--device", type=int, default=-1)
    args = ap.parse_args(argv)
    eng = Engine(device=args.device, autotune=True, use_graph=True)
    solvers = [EngineSolver(eng)]
    if args.plain:
        solvers.append(EngineSolver(eng, plain=True))
    out = run(solvers, args.problem_size, batch_sizes(args.initial, args.maximal, args.growth, args.rounds),
              args.csv, args.failed)
    eng.close()
    return 1 if out["failed"] is not None else 0


if __name__ == "__main__":
    raise SystemExit(main())

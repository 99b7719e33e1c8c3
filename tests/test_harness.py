"""Program.cs-style benchmark driver (sbfs/harness.py): batch-size schedule,
gpgpu.csv layout, reference seeds, and the cernyFailed.csv stop.

CPU tests drive the loop with stand-in solvers; the GPU test runs the engine
on two small rounds.
"""
import numpy as np
import pytest

from sbfs import dotnet_random as D
from sbfs import harness as H
from sbfs import problem as P


class _Recorder:
    def __init__(self, name, violation_at=None):
        self.name = name
        self.violation_at = violation_at
        self.seen = []

    def GetBestParallelism(self):
        return 2

    def verify_records(self, recs, n, lstride):
        self.seen.append((recs.shape[0], n, lstride, recs[:2].copy()))
        if self.violation_at is not None and recs.shape[0] >= self.violation_at[0]:
            return self.violation_at[1]
        return -1


def test_batch_sizes_follow_the_reference_loop():
    # Program.cs:76 with the commented-out 2^(1/8) growth
    s = H.batch_sizes(1 << 21, 1 << 25)
    assert s[0] == 1 << 21 and s[-1] < 1 << 25 and len(s) == 32
    assert s[8] in ((1 << 22) - 1, 1 << 22, (1 << 22) + 1)
    assert H.batch_sizes(10, 1000, 1.0, rounds=3) == [10, 10, 10]
    with pytest.raises(ValueError):
        H.batch_sizes(10, 100, 1.0)


def test_csv_rows_and_seeds(tmp_path):
    a, b = _Recorder("SolverA"), _Recorder("SolverB")
    csv, failed = str(tmp_path / "gpgpu.csv"), str(tmp_path / "cernyFailed.csv")
    out = H.run([a, b], 12, [300, 300, 500], csv, failed, log=lambda *_: None)
    text = open(csv).read()
    assert text == out["csv"]
    lines = text.split("\n")
    assert lines[0] == "problemsize,problemcount,SolverA,SolverB"
    assert [ln.split(",")[:2] for ln in lines[1:]] == [["12", "300"], ["12", "300"], ["12", "500"]]
    assert all(len(ln.split(",")) == 4 and int(ln.split(",")[2]) > 0 for ln in lines[1:])
    # each batch is FillArrayOfProblems(n, 12, 1234567 + n) in tight records
    count, n, lstride, head = a.seen[2]
    assert (count, n, lstride) == (500, 12, 12)
    np.testing.assert_array_equal(head, D.fill_array_of_problems(2, 12, 1234567 + 500, lstride=12))
    assert out["failed"] is None


def test_violation_is_appended_and_ends_the_run(tmp_path):
    a = _Recorder("SolverA", violation_at=(400, 7))
    csv, failed = str(tmp_path / "gpgpu.csv"), str(tmp_path / "cernyFailed.csv")
    out = H.run([a], 9, [200, 400, 800], csv, failed, log=lambda *_: None)
    assert out["failed"] == 7
    assert len(a.seen) == 2            # the 800 batch never runs
    recs = D.fill_array_of_problems(400, 9, 1234567 + 400, lstride=9)
    assert open(failed).read() == str(P.problems_from_records(recs[7:8], 9, 9)[0])
    assert open(csv).read().split("\n")[-1] == "9,400"


@pytest.mark.gpu
def test_engine_driver_rounds(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import sbfs
    with sbfs.Engine(device=0) as eng:
        solvers = [H.EngineSolver(eng), H.EngineSolver(eng, plain=True)]
        csv, failed = str(tmp_path / "gpgpu.csv"), str(tmp_path / "cernyFailed.csv")
        out = H.run(solvers, 12, [4096, 8192], csv, failed, log=lambda *_: None)
    assert out["failed"] is None
    lines = open(csv).read().split("\n")
    assert lines[0] == "problemsize,problemcount,SlimGPUNative,SlimGPUNativePlain"
    assert len(lines) == 3
    batched, plain = out["rates"][(8192, "SlimGPUNative")], out["rates"][(8192, "SlimGPUNativePlain")]
    assert batched > 20 * plain

"""Cerny-violation reporting (GPGPU/Program.cs:108-129): Verify over a batch,
then append the offending automaton's ToString() to cernyFailed.csv.

CPU tests drive the host logic with a stand-in IComputable; the GPU test
plants a "violation" by lowering the bound (sbfs_config.slack) so that C_9,
whose shortest word has (9-1)^2 = 64 letters, is reported.
"""
import numpy as np
import pytest

import sbfs
from sbfs import problem as P


class _FixedVerify:
    """IComputable stand-in whose Verify returns a fixed index."""

    def __init__(self, index):
        self.index = index
        self.calls = []

    def GetBestParallelism(self):
        return 3

    def Verify(self, problems, start, count, par):
        self.calls.append((start, count, par))
        return self.index


def test_report_appends_reference_format(tmp_path):
    probs = [P.generate_worst_case(5), P.Problem([1, 0, 2], [2, 2, 1], 3)]
    path = str(tmp_path / "cernyFailed.csv")
    solver = _FixedVerify(1)
    assert sbfs.verify_and_report(solver, probs, path) == 1
    assert solver.calls == [(0, 2, 3)]
    assert open(path).read() == "[[1,0,2],[2,2,1]]"
    # a second failure is appended without a separator, like File.AppendAllText
    assert sbfs.verify_and_report(_FixedVerify(0), probs, path) == 0
    assert open(path).read() == "[[1,0,2],[2,2,1]][[1,1,2,3,4],[1,2,3,4,0]]"
    back = sbfs.read_cerny_failed(path)
    assert [str(p) for p in back] == [str(probs[1]), str(probs[0])]


def test_no_report_when_bound_holds(tmp_path):
    path = tmp_path / "cernyFailed.csv"
    assert sbfs.verify_and_report(_FixedVerify(-1), [P.generate_worst_case(4)], str(path)) == -1
    assert not path.exists()


@pytest.mark.gpu
def test_planted_violation_is_reported(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sbfs import dotnet_random as D
    probs = P.problems_from_records(D.fill_array_of_problems(300, 9, 4321), 9)
    probs.insert(123, P.generate_worst_case(9))
    path = str(tmp_path / "cernyFailed.csv")
    with sbfs.Engine(slack=1) as eng:
        assert sbfs.verify_and_report(sbfs.SlimGPUNative(engine=eng), probs, path) == 123
    assert open(path).read() == str(P.generate_worst_case(9))
    with sbfs.Engine() as eng:
        assert sbfs.verify_and_report(sbfs.SlimGPUNative(engine=eng), probs, path) == -1
    assert len(sbfs.read_cerny_failed(path)) == 1

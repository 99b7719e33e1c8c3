"""The header-only C++ mirror of IComputable (include/sbfs_icomputable.hpp),
compiled with g++ against libsbfs.so and run as a separate program.

CPU: the program builds and its host-side pieces (GenerateWorstCase,
FillArrayOfProblems, ToString, the Verify.cs checks) agree with the Python
mirror.  GPU: Compute/Verify over a reference-seeded batch agree with the
oracle length for length.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import sbfs
from sbfs import dotnet_random as D
from sbfs import problem as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "icomputable_main.cpp")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ is not installed")
    lib_dir = os.path.dirname(sbfs.LIB_PATH)
    exe = str(tmp_path_factory.mktemp("cpp") / "icomputable_main")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-o", exe, sbfs.LIB_PATH, f"-Wl,-rpath,{lib_dir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_host_side(program):
    out = subprocess.run([program, "cpu"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.split()
    assert lines[0] == str(P.generate_worst_case(5))
    assert lines[1:4] == [str(p) for p in D.fill_array_of_problems_py(3, 13, 12456)]
    assert lines[4:] == ["cpu", "ok"]


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed,count", [(8, 10, 20000), (13, 12456, 20000), (18, 77, 400)])
def test_compute_matches_oracle(program, oracle_mod, n, seed, count):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    out = subprocess.run([program, "gpu", str(n), str(seed), str(count)], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    lens = np.array(out.stdout.split(), dtype=np.int32)
    recs = np.concatenate([D.fill_array_of_problems(count, n, seed), P.cerny_record(n)[None, :]])
    ref = oracle_mod.solve(recs, n=n, words=False, threads=8)
    np.testing.assert_array_equal(lens, ref["len"])

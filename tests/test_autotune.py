"""Autotuner: measured kernel shapes per size class, cached per device.

The tuned plan must keep results exact, and a second handle must pick the
cached choice up without measuring again."""
import time

import numpy as np
import pytest

import sbfs
from sbfs import problem as P

pytestmark = pytest.mark.gpu


def test_autotune_then_cache(tmp_path, oracle_mod):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cache = str(tmp_path / "tune.txt")
    t0 = time.perf_counter()
    with sbfs.Engine(device=0, autotune=True, tune_cache=cache) as eng:
        plan = eng.plan()
        first = time.perf_counter() - t0
        assert plan["tuned"] is True
        ns = P.uniform_sizes(20_000, 3, 20, 77)
        recs = P.uniform_maps(20_000, ns, 78)
        r = eng.solve(recs, ns=ns)
    ref = oracle_mod.solve(recs, ns=ns, words=False, threads=8)
    np.testing.assert_array_equal(r["len"], ref["len"])
    assert oracle_mod.replay(recs, r["len"], r["words"], ns=ns)[0] == 0
    text = open(cache).read()
    assert "c0=" in text and "c3=" in text
    t1 = time.perf_counter()
    with sbfs.Engine(device=0, autotune=True, tune_cache=cache) as eng2:
        plan2 = eng2.plan()
    assert plan2 == plan
    assert time.perf_counter() - t1 < first

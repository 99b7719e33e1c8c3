"""Serving loop (sbfs_server_*): continuous batching with admission control.

* every result equals the oracle's (lengths exact, words replay);
* a request gives the same length alone and in the mix (words may differ:
  shortest words are not unique, each must replay);
* malformed requests are refused at submission, a full queue refuses with
  SBFS_EBUSY, cancelling a pending request returns SBFS_ECANCELED;
* a mini-batch whose work failed completes its requests with SBFS_ECUDA, never
  with stale results, and so does every later request (the failure is made on
  the host: SBFS_SERVER_FAIL_BATCH reports one batch's event as failed).
"""
import os
import time

import numpy as np
import pytest

import sbfs
from sbfs import problem as P
from sbfs.server import Server

pytestmark = pytest.mark.gpu


def _requests(count, seed, lo=3, hi=22, cerny_every=20):
    ns = P.log_uniform_sizes(count, lo, hi, seed)
    recs = P.uniform_maps(count, ns, seed + 1)
    for i in range(0, count, cerny_every):
        recs[i] = P.cerny_record(int(ns[i]))
    return recs, ns


def _skip_without_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def test_serving_matches_oracle(oracle_mod):
    _skip_without_gpu()
    recs, ns = _requests(1500, 31, hi=24)   # the serving workload's sizes: up to n = 24
    with Server(device=0) as srv:
        ids = [srv.submit_record(recs[i], int(ns[i])) for i in range(len(ns))]
        res = srv.wait_all(ids)
        st = srv.stats()
    lens = np.array([res[i]["len"] for i in ids], dtype=np.int32)
    words = np.stack([res[i]["word"] for i in ids])
    ref = oracle_mod.solve(recs, ns=ns, words=False, threads=8)
    np.testing.assert_array_equal(lens, ref["len"])
    assert oracle_mod.replay(recs, lens, words, ns=ns)[0] == 0
    assert all(res[i]["status"] == 0 for i in ids)
    assert st["completed"] == len(ids) and st["small_batches"] >= 1 and st["level_launches"] >= 1
    assert st["arena_peak"] > 0


def test_alone_and_in_the_mix_agree(oracle_mod):
    _skip_without_gpu()
    recs, ns = _requests(400, 41, lo=6, hi=21, cerny_every=37)
    with Server(device=0) as srv:
        ids = [srv.submit_record(recs[i], int(ns[i])) for i in range(len(ns))]
        mix = srv.wait_all(ids)
        for i in range(0, len(ns), 23):
            rid = srv.submit_record(recs[i], int(ns[i]))
            alone = srv.wait_all([rid])[rid]
            assert alone["len"] == mix[ids[i]]["len"]
            L = alone["len"]
            if L > 0:
                assert oracle_mod.replay(recs[i:i + 1], np.array([L], dtype=np.int32), alone["word"][None, :],
                                         ns=ns[i:i + 1])[0] == 0


def test_admission_and_cancellation():
    _skip_without_gpu()
    a = np.array([1, 2, 0], dtype=np.uint8)
    with Server(device=0) as srv:
        with pytest.raises(sbfs.SbfsError) as ei:
            srv.submit(np.array([0, 5, 1], dtype=np.uint8), a, 3)   # state 5 in a 3-state automaton
        assert ei.value.status == 1
        assert not srv.cancel(123456789)
        assert srv.stats()["rejected"] == 1
    # a one-request queue with room for one large automaton: the rest must wait or be refused
    rec = P.cerny_record(22)
    fp = (1 << 22) // 8 + (1 << 22) * 8 + 512
    with Server(device=0, queue_capacity=1, arena_bytes=fp, max_levels=4) as srv:
        ids, busy = [], 0
        for _ in range(40):
            try:
                ids.append(srv.submit_record(rec, 22))
            except sbfs.SbfsError as e:
                assert e.status == 5   # SBFS_EBUSY
                busy += 1
        assert busy > 0
        cancelled = 0
        for rid in ids[1:]:
            cancelled += srv.cancel(rid)
        res = srv.wait_all(ids, timeout_s=300)
        done = [r for r in res.values() if r["status"] == 0]
        assert all(r["len"] == 21 * 21 for r in done)
        assert sum(r["status"] == 7 for r in res.values()) == cancelled
        assert srv.stats()["arena_peak"] <= fp


def test_failed_batch_completes_with_an_error_not_stale_results(oracle_mod):
    _skip_without_gpu()
    recs, ns = _requests(600, 57, lo=4, hi=16, cerny_every=50)
    os.environ["SBFS_SERVER_FAIL_BATCH"] = "2"
    try:
        srv = Server(device=0, max_batch=64)
    finally:
        del os.environ["SBFS_SERVER_FAIL_BATCH"]
    with srv:
        ids = [srv.submit_record(recs[i], int(ns[i])) for i in range(len(ns))]
        res = srv.wait_all(ids, timeout_s=120)
        late = [srv.submit_record(recs[i], int(ns[i])) for i in range(5)]
        late_res = srv.wait_all(late, timeout_s=60)
    status = np.array([res[i]["status"] for i in ids])
    assert set(status.tolist()) <= {0, 4} and (status == 4).sum() > 0
    ok = np.nonzero(status == 0)[0]
    ref = oracle_mod.solve(recs, ns=ns, words=False, threads=8)
    got = np.array([res[ids[i]]["len"] for i in ok], dtype=np.int32)
    np.testing.assert_array_equal(got, ref["len"][ok])
    assert all(res[ids[i]]["len"] == -1 for i in np.nonzero(status == 4)[0])
    assert all(r["status"] == 4 for r in late_res.values())


def test_submit_many_and_the_small_footprint_budget(oracle_mod):
    """Requests submitted in one call come back exactly as the oracle has them,
    and the n <= 20 mini-batches never hold more than their footprint budget
    (2^n / 8 + 64 bytes per request in flight)."""
    _skip_without_gpu()
    recs, ns = _requests(3000, 71, lo=3, hi=20, cerny_every=40)
    budget = 4 << 20
    with Server(device=0, small_budget_bytes=budget) as srv:
        bad = recs[:3].copy()
        bad[1, 0] = 63                            # state 63 in a small automaton: malformed
        with pytest.raises(sbfs.SbfsError) as ei:
            srv.submit_many(bad, ns[:3])
        assert ei.value.status == 1
        ids = srv.submit_many(recs, ns)
        res = srv.wait_all(ids.tolist(), timeout_s=120)
        st = srv.stats()
    lens = np.array([res[int(i)]["len"] for i in ids], dtype=np.int32)
    words = np.stack([res[int(i)]["word"] for i in ids])
    ref = oracle_mod.solve(recs, ns=ns, words=False, threads=8)
    np.testing.assert_array_equal(lens, ref["len"])
    assert oracle_mod.replay(recs, lens, words, ns=ns)[0] == 0
    assert 0 < st["small_peak"] <= budget and st["small_used"] == 0
    assert st["small_batches"] > 1                # the budget split the burst into several mini-batches
    assert st["rejected"] == 3

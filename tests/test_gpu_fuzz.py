"""Randomised parity: seeded batches of many shapes through every entry point,
against the oracle.

Each case draws a batch shape from its seed: batch size (including empty and
single-automaton batches), one n for the batch or a per-automaton n, record
stride (tight, padded, 64-byte), and a sprinkling of special members --
Cerny automata, permutation-plus-merge, pairs of permutations (never
synchronizing), constant maps (length 1), identities and n = 1.  The batch
then goes through sbfs_solve_batch (host buffers, words on or off),
sbfs_verify_batch, a small-chunk handle (the multi-stream chunked path) and
sbfs_solve_batch_device (device buffers).  Lengths and flags must be
bit-exact; every word must replay to a singleton in its length.
"""
import numpy as np
import pytest

import sbfs
from sbfs import problem as P

pytestmark = pytest.mark.gpu

COUNTS = [0, 1, 2, 31, 33, 257, 1000, 4099, 20_000, 70_001]


def _case(seed):
    rng = np.random.default_rng(10_007 + seed)
    count = int(rng.choice(COUNTS))
    mixed = bool(rng.integers(0, 2))
    if mixed:
        lo = int(rng.integers(1, 21))
        hi = int(rng.integers(lo, 23))
        ns = rng.integers(lo, hi + 1, size=count).astype(np.uint8)
        max_n = int(ns.max()) if count else hi
    else:
        n = int(rng.integers(1, 23))
        ns = np.full(count, n, dtype=np.uint8)
        max_n = n
    lstride = int(rng.choice([max_n, min(32, max_n + 1 + int(rng.integers(0, 4))), 32]))
    lstride = max(lstride, max_n)
    recs = P.uniform_maps(count, ns if count else 1, 77 * seed + 5, lstride=lstride) if count else \
        np.zeros((0, 2 * lstride), np.uint8)
    # special members, a few percent of the batch
    for i in rng.choice(count, size=min(count, 1 + count // 40), replace=False) if count else []:
        n = int(ns[i])
        kind = int(rng.integers(0, 5))
        rec = np.zeros(2 * lstride, np.uint8)
        if kind == 0 and 2 <= n <= 20:
            rec = P.cerny_record(n, lstride)
        elif kind == 1 and n >= 2:
            rec = P.perm_merge_record(n, int(rng.integers(0, 1 << 30)), lstride)
        elif kind == 2:
            rec[:n] = rng.permutation(n)
            rec[lstride:lstride + n] = rng.permutation(n)
        elif kind == 3:
            rec[:n] = int(rng.integers(0, n))
            rec[lstride:lstride + n] = rng.integers(0, n, size=n)
        else:
            rec[:n] = np.arange(n)
            rec[lstride:lstride + n] = np.arange(n)
        recs[i] = rec
    if mixed:
        return recs, ns, 0, lstride, rng
    return recs, None, (int(ns[0]) if count else max_n), lstride, rng


@pytest.fixture(scope="module")
def chunked():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    eng = sbfs.Engine(device=0, chunk=1 << 12)
    yield eng
    eng.close()


@pytest.mark.parametrize("seed", range(24))
def test_fuzz_parity(engine, chunked, oracle_mod, seed):
    import torch
    recs, ns, n, lstride, rng = _case(seed)
    count = recs.shape[0]
    ref = oracle_mod.solve(recs, ns=ns, n=n, lstride=lstride, words=False, threads=8)
    words = bool(rng.integers(0, 4))          # mostly with words
    r = engine.solve(recs, ns=ns, n=n, lstride=lstride, words=words)
    np.testing.assert_array_equal(r["len"], ref["len"])
    assert r["first_violation"] == ref["first_violation"]
    if words and count:
        assert oracle_mod.replay(recs, r["len"], r["words"], ns=ns, n=n, lstride=lstride)[0] == 0
    v = engine.verify(recs, ns=ns, n=n, lstride=lstride)
    np.testing.assert_array_equal(v["len"], ref["len"])
    c = chunked.solve(recs, ns=ns, n=n, lstride=lstride)
    np.testing.assert_array_equal(c["len"], ref["len"])
    if count:
        assert oracle_mod.replay(recs, c["len"], c["words"], ns=ns, n=n, lstride=lstride)[0] == 0
        # device-resident buffers
        dev = torch.device("cuda", 0)
        ws = r["word_stride"]
        d_maps = torch.from_numpy(recs).to(dev)
        d_ns = torch.from_numpy(ns).to(dev) if ns is not None else None
        d_len = torch.full((count,), -7, dtype=torch.int32, device=dev)
        d_words = torch.zeros((count, ws), dtype=torch.int64, device=dev)
        d_fv = torch.zeros(1, dtype=torch.int64, device=dev)
        max_n = int(ns.max()) if ns is not None else n
        engine.solve_device(d_maps, lstride, count, n=n, d_ns=d_ns, max_n=max_n, d_len=d_len, d_words=d_words,
                            word_stride=ws, d_first_violation=d_fv)
        engine.wait_device()
        lens = d_len.cpu().numpy()
        np.testing.assert_array_equal(lens, ref["len"])
        assert int(d_fv.item()) == ref["first_violation"]
        wd = d_words.cpu().numpy().view(np.uint64)
        assert oracle_mod.replay(recs, lens, wd, ns=ns, n=n, lstride=lstride)[0] == 0

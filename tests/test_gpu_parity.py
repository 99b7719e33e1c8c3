"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Bar: every length and non-synchronizing flag bit-exact; every returned word
replays to a singleton and has the returned length; the Cerny bound (n-1)^2 is
checked per automaton (Verify.cs:12-62).  Sizes follow the benchmark
configurations with seeded synthetic inputs.
"""
import os

import numpy as np
import pytest

import sbfs
from sbfs import problem as P

pytestmark = pytest.mark.gpu


def _check(oracle_mod, recs, r, ns=None, n=0, lstride=32, ref=None):
    if ref is None:
        ref = oracle_mod.solve(recs, ns=ns, n=n, lstride=lstride, words=False, threads=8)
    np.testing.assert_array_equal(r["len"], ref["len"])
    if "stats" in r:
        assert r["stats"]["synchronizing"] == int((ref["len"] >= 0).sum())
    if r.get("words") is not None:
        bad, ok = oracle_mod.replay(recs, r["len"], r["words"], ns=ns, n=n, lstride=lstride)
        assert bad == 0, np.nonzero(ok != 3)[0][:10]
    assert r["first_violation"] == ref["first_violation"] == -1
    return ref


def test_config1_plain_n8(engine, oracle_mod):
    recs = P.uniform_maps(10_000, 8, 0x5EED + 0)
    r = engine.solve(recs, n=8)
    ref = _check(oracle_mod, recs, r, n=8)
    assert (r["len"] > 49).sum() == 0
    # the GPU finishes the step in which the first singleton appears while the
    # sequential oracle stops at that singleton (more expansions), but a warp
    # sharing one heavy automaton may meet a singleton earlier within the last
    # level than the sequential order does (fewer): the totals stay close
    ratio = r["stats"]["expanded"] / ref["expanded"]
    assert 0.95 <= ratio <= 1.5, ratio


def test_config2_n12_full_batch_and_sample(engine, oracle_mod):
    recs = P.uniform_maps(1_000_000, 12, 0x5EED + 1)
    r = engine.solve(recs, n=12)
    sample = slice(0, None, 100)
    ref_s = oracle_mod.solve(recs[sample], n=12, words=False)
    np.testing.assert_array_equal(r["len"][sample], ref_s["len"])
    _check(oracle_mod, recs, r, n=12)


@pytest.mark.parametrize("seed", range(12456, 12466))
def test_reference_integrity_batches(engine, oracle_mod, seed):
    """AlgorithmCorrectnessTestProject/IntegrityTest.cs:62-87: 2^17 automata of
    13 states from Problem.FillArrayOfProblems with seeds 12456..12465."""
    from sbfs import dotnet_random as D
    recs = D.fill_array_of_problems(1 << 17, 13, seed, lstride=13)
    r = engine.solve(recs, n=13, lstride=13)
    _check(oracle_mod, recs, r, n=13, lstride=13)


def test_reference_benchmark_batch(engine, oracle_mod):
    """The batch GPGPU/Program.cs:94 times for 2^20 automata at n = 12 (seed
    1234567 + 2^20), in tight 24-byte records."""
    from sbfs import dotnet_random as D
    count = 1 << 20
    recs = D.benchmark_batch(count, 12, lstride=12)
    r = engine.solve(recs, n=12, lstride=12)
    _check(oracle_mod, recs, r, n=12, lstride=12)
    v = engine.verify(recs, n=12, lstride=12)
    np.testing.assert_array_equal(v["len"], r["len"])
    assert v["first_violation"] == -1


def test_tight_records_same_as_64_byte_records(engine):
    recs = P.uniform_maps(50_000, 12, 42)
    a = engine.solve(recs, n=12, words=False)
    b = engine.solve(P.repack(recs, 32, 12), n=12, lstride=12, words=False)
    np.testing.assert_array_equal(a["len"], b["len"])


@pytest.mark.parametrize("n", [3, 5, 8, 9, 12, 13, 14, 16, 17, 20, 21, 24])
def test_cerny_known_answers(engine, n):
    recs = np.stack([P.cerny_record(n)] * 3)
    r = engine.solve(recs, n=n)
    assert (r["len"] == (n - 1) ** 2).all()


def test_reference_worst_case_letters(engine, oracle_mod):
    probs = [P.generate_worst_case(n) for n in range(3, 14)]
    recs, ns = P.records_from_problems(probs)
    r = engine.solve(recs, ns=ns)
    assert list(r["len"]) == [(n - 1) ** 2 for n in range(3, 14)]
    bad, _ = oracle_mod.replay(recs, r["len"], r["words"], ns=ns)
    assert bad == 0


@pytest.mark.parametrize("n", [4, 6, 10, 14, 16, 18, 20])
def test_uniform_random_each_class(engine, oracle_mod, n):
    cnt = 20_000 if n <= 16 else 2_000
    recs = P.uniform_maps(cnt, n, 1000 + n)
    r = engine.solve(recs, n=n)
    _check(oracle_mod, recs, r, n=n)


def test_mixed_sizes_with_cerny(engine, oracle_mod):
    cnt = 20_000
    ns = P.uniform_sizes(cnt, 6, 20, 0x5EED + 2)
    recs = P.uniform_maps(cnt, ns, 0x5EED + 2)
    idx = np.arange(0, cnt, 100)  # 1% Cerny
    for i in idx:
        recs[i] = P.cerny_record(int(ns[i]))
    r = engine.solve(recs, ns=ns)
    _check(oracle_mod, recs, r, ns=ns)
    np.testing.assert_array_equal(r["len"][idx], (ns[idx].astype(np.int32) - 1) ** 2)


def test_alone_equals_in_the_mix(engine):
    ns = P.uniform_sizes(3000, 6, 22, 11)
    recs = P.uniform_maps(3000, ns, 12)
    mix = engine.solve(recs, ns=ns)
    for i in range(0, 3000, 211):
        one = engine.solve(recs[i:i + 1], ns=ns[i:i + 1])
        assert one["len"][0] == mix["len"][i]


def test_plain_form_matches_batched(engine):
    recs = P.uniform_maps(300, 12, 77)
    a = engine.solve(recs, n=12)
    b = engine.solve(recs, n=12, plain=True)
    np.testing.assert_array_equal(a["len"], b["len"])


def test_verify_mode_and_slack(oracle_mod):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    recs = np.stack([P.uniform_maps(1, 9, 1)[0]] * 5 + [P.cerny_record(9)] + [P.uniform_maps(1, 9, 2)[0]])
    with sbfs.Engine(slack=1) as eng:
        v = eng.verify(recs, n=9)
        assert v["first_violation"] == 5
        assert v["len"][5] == 64
    with sbfs.Engine() as eng:
        assert eng.verify(recs, n=9, lengths=False)["first_violation"] == -1


def test_pinned_and_pageable_buffers_agree(engine, oracle_mod):
    import torch
    recs = P.uniform_maps(70_000, 12, 5)
    a = engine.solve(recs, n=12)
    pin = torch.from_numpy(recs).pin_memory()
    out_len = torch.empty(recs.shape[0], dtype=torch.int32).pin_memory()
    out_words = torch.empty((recs.shape[0], 2), dtype=torch.int64).pin_memory()
    b = engine.solve(pin.numpy(), n=12, out=(out_len.numpy(), out_words.numpy().view(np.uint64)))
    np.testing.assert_array_equal(a["len"], b["len"])
    # a shortest word need not be unique; which one comes back may differ
    # between runs, every one must replay to a singleton
    for r in (a, b):
        assert oracle_mod.replay(recs, r["len"], r["words"], n=12)[0] == 0


def test_malformed_automaton_is_rejected(engine):
    recs = P.uniform_maps(100, 8, 3)
    recs[17, 2] = 8  # state 8 in an 8-state automaton
    with pytest.raises(sbfs.SbfsError) as ei:
        engine.solve(recs, n=8)
    assert ei.value.status == 1
    # the handle stays usable
    good = engine.solve(P.uniform_maps(10, 8, 3), n=8)
    assert good["len"].shape == (10,)


def test_empty_batch(engine):
    r = engine.solve(np.zeros((0, 64), dtype=np.uint8), n=8)
    assert r["len"].shape == (0,) and r["first_violation"] == -1


def test_icomputable_mirror(engine, oracle_mod):
    probs = P.problems_from_records(P.uniform_maps(500, 10, 8), 10)
    solver = sbfs.SlimGPUNative(engine=engine)
    results = [None] * 510
    assert solver.Compute(probs, 0, results, 10, 500, solver.GetBestParallelism()) == -1
    recs, ns = P.records_from_problems(probs)
    ref = oracle_mod.solve(recs, ns=ns, words=False)
    for i in range(500):
        res = results[10 + i]
        assert res.isSynchronizable == (ref["len"][i] >= 0)
        if res.isSynchronizable:
            assert res.shortestSynchronizingWordLength == ref["len"][i]
            assert len(res.shortestSynchronizingWord) == ref["len"][i]
    assert solver.Verify(probs, 0, 500, 1) == -1


def test_device_buffer_path(engine, oracle_mod):
    import torch
    ns = P.uniform_sizes(30_000, 3, 20, 21)
    recs = P.uniform_maps(30_000, ns, 22)
    dev = torch.device("cuda", 0)
    d_maps = torch.from_numpy(recs).to(dev)
    d_ns = torch.from_numpy(ns).to(dev)
    d_len = torch.empty(len(ns), dtype=torch.int32, device=dev)
    d_words = torch.empty((len(ns), 6), dtype=torch.int64, device=dev)
    d_fv = torch.empty(1, dtype=torch.int64, device=dev)
    s = torch.cuda.Stream()
    engine.solve_device(d_maps, 32, len(ns), d_ns=d_ns, max_n=20, d_len=d_len, d_words=d_words,
                        word_stride=6, d_first_violation=d_fv, stream=s)
    st = engine.wait_device()
    assert st["automata"] == len(ns) and st["launches"] >= 3
    lens = d_len.cpu().numpy()
    assert st["synchronizing"] == int((lens >= 0).sum())
    ref = oracle_mod.solve(recs, ns=ns, words=False, threads=8)
    np.testing.assert_array_equal(lens, ref["len"])
    assert int(d_fv.item()) == -1
    words = d_words.cpu().numpy().view(np.uint64)
    assert oracle_mod.replay(recs, lens, words, ns=ns)[0] == 0
    # the host path on the same handle afterwards still agrees
    host = engine.solve(recs, ns=ns)
    np.testing.assert_array_equal(host["len"], lens)


def test_cuda_graph_replay_matches(oracle_mod):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    recs = P.uniform_maps(120_000, 12, 901)
    ns = P.uniform_sizes(50_000, 3, 18, 902)
    mixed = P.uniform_maps(50_000, ns, 903)
    ref = oracle_mod.solve(recs, n=12, words=False, threads=8)["len"]
    ref_mixed = oracle_mod.solve(mixed, ns=ns, words=False, threads=8)["len"]
    with sbfs.Engine(device=0, use_graph=True, chunk=1 << 16) as eng:
        for rep in range(4):        # direct, captured, then replayed twice
            r = eng.solve(recs, n=12)
            np.testing.assert_array_equal(r["len"], ref)
            assert oracle_mod.replay(recs, r["len"], r["words"], n=12)[0] == 0
            m = eng.solve(mixed, ns=ns)
            np.testing.assert_array_equal(m["len"], ref_mixed)
            assert r["stats"]["synchronizing"] == int((ref >= 0).sum())
            assert m["stats"]["synchronizing"] == int((ref_mixed >= 0).sum())
        big = P.uniform_maps(300_000, 12, 904)   # larger chunks: buffers move, graphs rebuild
        with sbfs.Engine(device=0, use_graph=True, chunk=1 << 18) as eng2:
            for rep in range(3):
                rb = eng2.solve(big, n=12)
                rs = eng2.solve(recs, n=12)
                np.testing.assert_array_equal(rs["len"], ref)
        np.testing.assert_array_equal(rb["len"], oracle_mod.solve(big, n=12, words=False, threads=8)["len"])
        dev = torch.device("cuda", 0)
        d_maps = torch.from_numpy(recs).to(dev)
        d_len = torch.empty(len(recs), dtype=torch.int32, device=dev)
        d_words = torch.empty((len(recs), 2), dtype=torch.int64, device=dev)
        d_fv = torch.empty(1, dtype=torch.int64, device=dev)
        s = torch.cuda.Stream()
        for rep in range(4):
            d_len.fill_(-9)
            torch.cuda.synchronize()
            eng.solve_device(d_maps, 32, len(recs), n=12, d_len=d_len, d_words=d_words, word_stride=2,
                             d_first_violation=d_fv, stream=s)
            eng.wait_device()
            np.testing.assert_array_equal(d_len.cpu().numpy(), ref)


def test_level_slots_recycle_under_load(oracle_mod):
    """More n=21 automata than level slots, with long (Cerny) and short ones
    mixed, so slots finish, are freed and re-admitted while others run."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    recs = P.uniform_maps(600, 21, 1234)
    for i in range(0, 600, 97):
        recs[i] = P.cerny_record(21)
    with sbfs.Engine(device=0) as eng:
        r = eng.solve(recs, n=21)
    ref = oracle_mod.solve(recs, n=21, words=False, threads=16)
    np.testing.assert_array_equal(r["len"], ref["len"])
    assert oracle_mod.replay(recs, r["len"], r["words"], n=21)[0] == 0


@pytest.mark.parametrize("n,count", [(12, 300_001), (8, 262_145), (11, 1_000_003), (13, 300_007), (14, 262_151)])
def test_streamed_host_path(oracle_mod, n, count):
    """Uniform n <= 14 batches of at least two 2^17-automaton chunks take the
    streamed host path (one kernel, chunked copies both ways, escalated
    automata patched in at the end); an explicit chunk size takes the
    chunked multi-stream path.  Both must match the oracle."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sbfs import dotnet_random as D
    recs = D.fill_array_of_problems(count, n, 777 + n, lstride=n)
    if n >= 13:
        # Cerny C_13 / C_14 members: 144- and 169-letter words, three 64-bit words
        # through the escalation patch
        for i in (5, 150_001, count - 1):
            recs[i] = P.repack(P.cerny_record(n)[None, :], 32, n)[0]
    ref = oracle_mod.solve(recs, n=n, lstride=n, words=False, threads=8)
    if n >= 13:
        assert ref["len"][150_001] == (n - 1) ** 2
    with sbfs.Engine(device=0) as eng, sbfs.Engine(device=0, chunk=1 << 16) as chunked:
        r = eng.solve(recs, n=n, lstride=n)
        _check(oracle_mod, recs, r, n=n, lstride=n, ref=ref)
        # the streamed path: one BFS kernel, the result count, the escalated-result patch
        assert r["stats"]["launches"] <= 3
        # pinned host buffers (direct copies) give the same lengths; words replay
        pin = torch.from_numpy(recs).pin_memory()
        out_len = torch.empty(count, dtype=torch.int32).pin_memory()
        out_words = torch.empty((count, r["word_stride"]), dtype=torch.int64).pin_memory()
        p = eng.solve(pin.numpy(), n=n, lstride=n, out=(out_len.numpy(), out_words.numpy().view(np.uint64)))
        np.testing.assert_array_equal(p["len"], ref["len"])
        assert oracle_mod.replay(recs, p["len"], p["words"], n=n, lstride=n)[0] == 0
        # one side pinned, the other pageable: pageable results are staged chunk by
        # chunk and the escalated automata's results written by the host
        q = eng.solve(pin.numpy(), n=n, lstride=n)
        np.testing.assert_array_equal(q["len"], ref["len"])
        assert oracle_mod.replay(recs, q["len"], q["words"], n=n, lstride=n)[0] == 0
        if n >= 11:
            assert q["stats"]["escalated"] > 0
        out_len.zero_()
        out_words.zero_()
        q = eng.solve(recs, n=n, lstride=n, out=(out_len.numpy(), out_words.numpy().view(np.uint64)))
        np.testing.assert_array_equal(q["len"], ref["len"])
        assert oracle_mod.replay(recs, q["len"], q["words"], n=n, lstride=n)[0] == 0
        v = eng.verify(recs, n=n, lstride=n)
        np.testing.assert_array_equal(v["len"], ref["len"])
        assert eng.verify(recs, n=n, lstride=n, lengths=False)["first_violation"] == -1
        c = chunked.solve(recs, n=n, lstride=n)
        np.testing.assert_array_equal(c["len"], ref["len"])
        assert c["stats"]["launches"] > 3


def test_streamed_path_violation_and_malformed(oracle_mod):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from sbfs import dotnet_random as D
    count = 400_000
    recs = D.fill_array_of_problems(count, 12, 4242, lstride=12)
    recs[333_333] = P.repack(P.cerny_record(12)[None, :], 32, 12)[0]
    with sbfs.Engine(device=0, slack=1) as eng:
        v = eng.verify(recs, n=12, lstride=12)
        assert v["first_violation"] == 333_333 and v["len"][333_333] == 121
    bad = recs.copy()
    bad[299_999, 3] = 12   # state 12 in a 12-state automaton
    bad[123_456, 20] = 200   # b(8) = 200: far out of range
    out_len = np.zeros(count, dtype=np.int32)
    out_words = np.zeros((count, 2), dtype=np.uint64)
    with sbfs.Engine(device=0) as eng:
        with pytest.raises(sbfs.SbfsError) as ei:
            eng.solve(bad, n=12, lstride=12, out=(out_len, out_words))
        assert ei.value.status == 1
        assert out_len[299_999] == -2 and out_len[123_456] == -2
        assert (out_len >= -1).sum() == count - 2
        r = eng.solve(recs, n=12, lstride=12)   # the handle stays usable
        assert r["first_violation"] == -1 and r["len"][333_333] == 121


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_automata.npz")


def test_golden_fixtures_on_every_small_path(engine):
    """The committed fixtures (lengths from word enumeration, not from a BFS):
    n = 2 and 3 exhaustive, n = 4..6 seeded; per-lane, warp-pooled and plain."""
    d = np.load(GOLDEN)
    recs, ns, lens = d["recs"], d["ns"], d["lens"]
    np.testing.assert_array_equal(engine.solve(recs, ns=ns)["len"], lens)
    with sbfs.Engine(device=0, small_kernel=2) as pooled:
        np.testing.assert_array_equal(pooled.solve(recs, ns=ns)["len"], lens)
    few = slice(0, None, 40)
    np.testing.assert_array_equal(engine.solve(recs[few], ns=ns[few], plain=True)["len"], lens[few])


def test_one_state_automata_match_the_oracle(engine, oracle_mod):
    recs = np.zeros((4, 64), dtype=np.uint8)   # n = 1: both letters map state 0 to itself
    r = engine.solve(recs, n=1)
    ref = oracle_mod.solve(recs, n=1, words=False)
    np.testing.assert_array_equal(r["len"], ref["len"])


def test_largest_sizes(engine, oracle_mod):
    """n = 25..28 (2^28-bit bitmaps in the level slots), the Cerny automaton at
    the maximum size, and a slowly synchronizing permutation + merge."""
    ns = np.array([25, 26, 27, 28, 28, 28, 24], dtype=np.uint8)
    rows = [P.uniform_maps(1, int(n), 900 + i)[0] for i, n in enumerate(ns[:-3])]
    rows += [P.cerny_record(28), P.uniform_maps(1, 28, 999)[0], P.perm_merge_record(24, 7)]
    recs = np.stack(rows)
    r = engine.solve(recs, ns=ns)
    assert r["len"][4] == 27 * 27
    check = [0, 1, 2, 3, 5, 6]
    ref = oracle_mod.solve(recs[check], ns=ns[check], words=False, threads=8)
    np.testing.assert_array_equal(r["len"][check], ref["len"])
    assert oracle_mod.replay(recs, r["len"], r["words"], ns=ns)[0] == 0
    assert r["first_violation"] == -1


def _two_component_record(n, seed):
    """States 0..h-1 and h..n-1 each closed under both letters: never synchronizing,
    with a wide reachable power set (pairs of subsets of the two halves)."""
    h = n // 2
    rec = np.zeros(2 * P.RECORD_LSTRIDE, dtype=np.uint8)
    lo = P.uniform_maps(1, h, seed)[0]
    hi = P.uniform_maps(1, n - h, seed + 1)[0]
    for letter in range(2):
        base = letter * P.RECORD_LSTRIDE
        rec[base:base + h] = lo[base:base + h]
        rec[base + h:base + n] = hi[base:base + n - h] + h
    return rec


def test_n17_20_hash_set_path_and_hand_offs(engine, oracle_mod):
    """n = 17..20: one warp per automaton with a hash set; Cerny automata (past the
    level cap), slow permutation + merge automata and two-component automata
    (wide, never synchronizing) go on to the CTA-wide kernel."""
    cnt = 40_000
    ns = P.uniform_sizes(cnt, 17, 20, 0x5EED + 17)
    recs = P.uniform_maps(cnt, ns, 0x5EED + 17)
    cerny = np.arange(3, cnt, 500)
    slow = np.arange(5, cnt, 777)
    wide = np.arange(7, cnt, 997)
    for i in cerny:
        recs[i] = P.cerny_record(int(ns[i]))
    for i in slow:
        recs[i] = P.perm_merge_record(int(ns[i]), int(i))
    for i in wide:
        recs[i] = _two_component_record(int(ns[i]), int(i))
    r = engine.solve(recs, ns=ns)
    _check(oracle_mod, recs, r, ns=ns)
    np.testing.assert_array_equal(r["len"][cerny], (ns[cerny].astype(np.int32) - 1) ** 2)
    assert (r["len"][wide] == -1).all()
    # a malformed member is rejected, and the handle stays usable
    bad = recs[:64].copy()
    bad[40, P.RECORD_LSTRIDE + 3] = ns[40]
    with pytest.raises(sbfs.SbfsError) as ei:
        engine.solve(bad, ns=ns[:64])
    assert ei.value.status == 1
    np.testing.assert_array_equal(engine.solve(recs[:64], ns=ns[:64])["len"], r["len"][:64])


def test_n13_16_hash_set_and_pooled_paths(engine, oracle_mod):
    """n = 13..16 on the hash-set warps (default) and on the warp-pooled kernel
    (small_kernel=2), Cerny members handed to the CTA-wide kernel on both."""
    cnt = 30_000
    ns = P.uniform_sizes(cnt, 13, 16, 0x5EED + 13)
    recs = P.uniform_maps(cnt, ns, 0x5EED + 13)
    cerny = np.arange(11, cnt, 300)
    for i in cerny:
        recs[i] = P.cerny_record(int(ns[i]))
    ref = oracle_mod.solve(recs, ns=ns, words=False, threads=8)
    _check(oracle_mod, recs, engine.solve(recs, ns=ns), ns=ns, ref=ref)
    with sbfs.Engine(device=0, small_kernel=2) as pooled:
        _check(oracle_mod, recs, pooled.solve(recs, ns=ns), ns=ns, ref=ref)
    assert (ref["len"][cerny] == (ns[cerny].astype(np.int32) - 1) ** 2).all()


def test_permutation_automata_on_every_class(engine, oracle_mod):
    """Both letters permutations never synchronize: the full set maps to itself
    under both letters.  One batch spans every size class (n = 2..24)."""
    rng = np.random.default_rng(12)
    ns = np.array([2, 5, 8, 9, 12, 13, 16, 17, 20, 21, 24] * 3, dtype=np.uint8)
    recs = np.zeros((len(ns), 64), dtype=np.uint8)
    for i, n in enumerate(ns):
        recs[i, :n] = rng.permutation(int(n))
        recs[i, 32:32 + n] = rng.permutation(int(n))
    r = engine.solve(recs, ns=ns)
    assert (r["len"] == -1).all()
    np.testing.assert_array_equal(r["len"], oracle_mod.solve(recs, ns=ns, words=False)["len"])


def test_bounded_device_wait_runs_out_and_the_handle_recovers(oracle_mod):
    """The streamed host path's kernel waits, bounded, for each chunk of records
    to arrive.  Withhold one chunk's ready flag (a host-side hook: the records
    still arrive, the flag does not) with a short poll limit: the wait runs out,
    the call returns SBFS_ETIMEOUT, and the same handle then solves the next
    batch exactly."""
    import os
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    count, n = 1 << 19, 12                     # four 2^17 chunks: the streamed path
    recs = P.repack(P.uniform_maps(count, n, 0xB0B), 32, n)
    os.environ["SBFS_TEST_SKIP_CHUNK_READY"] = "2"
    try:
        eng = sbfs.Engine(device=0, wait_polls=1 << 12)   # about 1 ms of polls
    finally:
        del os.environ["SBFS_TEST_SKIP_CHUNK_READY"]
    with eng:
        with pytest.raises(sbfs.SbfsError) as ei:
            eng.solve(recs, n=n, lstride=n)
        assert ei.value.status == 3            # SBFS_ETIMEOUT
        r = eng.solve(recs, n=n, lstride=n)
    ref = oracle_mod.solve(recs, n=n, lstride=n, words=False, threads=8)
    np.testing.assert_array_equal(r["len"], ref["len"])
    assert oracle_mod.replay(recs, r["len"], r["words"], n=n, lstride=n)[0] == 0


def test_config3_mixed_full_batch_as_benchmarked(engine, oracle_mod):
    """The mixed configuration exactly as bench.py times it: 200,000 automata,
    n uniform in 6..20, 1 % Cerny family (expected length (n-1)^2); every
    length against the oracle, every word replayed."""
    import bench
    wl = bench.make_workload("mixed")
    assert wl["count"] == 200_000
    r = engine.solve(wl["recs"], ns=wl["ns"], lstride=32)
    ref = _check(oracle_mod, wl["recs"], r, ns=wl["ns"])
    cerny = np.arange(0, wl["count"], 100)
    np.testing.assert_array_equal(r["len"][cerny], (wl["ns"][cerny].astype(np.int32) - 1) ** 2)
    assert ref["len"].max() == 19 * 19


def test_config5_large_instances_as_named(engine, oracle_mod):
    """The large configuration exactly as named: n = 24, 26, 28, each with 64
    uniform random automata, the Cerny automaton C_n and a random permutation
    plus one merge; every length against the oracle (which runs the same
    power-set BFS on the host), every word replayed."""
    import bench
    wl = bench.make_workload("large")
    assert wl["count"] == 3 * 66
    r = engine.solve(wl["recs"], ns=wl["ns"], lstride=32)
    ref = _check(oracle_mod, wl["recs"], r, ns=wl["ns"])
    for n in (24, 26, 28):
        idx = np.nonzero(wl["ns"] == n)[0]
        assert r["len"][idx[64]] == (n - 1) ** 2              # C_n
    assert (ref["len"] >= 0).sum() > 100


def test_streamed_batch_as_a_fresh_process_first_call(oracle_mod, tmp_path):
    """A process whose very first call is a streamed batch (uniform n <= 12, at
    least 2^18 automata, pageable buffers): the kernel runs while the records
    stream in, so nothing the host launches behind it may wait for the device
    to go idle (a kernel's first launch loads its module).  Run in a fresh
    child process, so that no earlier call has loaded any kernel."""
    import subprocess
    import sys
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    count, n = 1 << 19, 12
    recs = P.uniform_maps(count, n, 0xF1257)
    np.save(tmp_path / "recs.npy", recs)
    pkg = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "gpgpu-binary-automaton-synchronizing-algorithms_b200")
    code = ("import sys, numpy as np; sys.path.insert(0, sys.argv[1]); import sbfs; "
            "r = np.load(sys.argv[2]); e = sbfs.Engine(device=0); out = e.solve(r, n=12); "
            "np.save(sys.argv[3], out['len']); np.save(sys.argv[4], out['words'])")
    res = subprocess.run([sys.executable, "-c", code, pkg, str(tmp_path / "recs.npy"), str(tmp_path / "len.npy"),
                          str(tmp_path / "words.npy")], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    lens = np.load(tmp_path / "len.npy")
    words = np.load(tmp_path / "words.npy")
    ref = oracle_mod.solve(recs, n=n, words=False, threads=8)
    np.testing.assert_array_equal(lens, ref["len"])
    assert oracle_mod.replay(recs, lens, words, n=n)[0] == 0


def test_equal_sizes_take_the_uniform_path(engine, oracle_mod):
    """A per-automaton size array whose entries are all equal (the IComputable
    mirrors always pass one) runs as a uniform batch: no size bytes cross the
    link, and the results equal those of the same batch given one n."""
    count, n = 50_000, 13
    recs = P.uniform_maps(count, n, 0x5A5A)
    recs[7] = P.cerny_record(n)
    ns = np.full(count, n, dtype=np.uint8)
    r = engine.solve(recs, ns=ns)
    assert r["stats"]["h2d_bytes"] == count * 64           # records only
    u = engine.solve(recs, n=n)
    np.testing.assert_array_equal(r["len"], u["len"])
    ref = _check(oracle_mod, recs, r, ns=ns)
    assert ref["len"][7] == (n - 1) ** 2
    # one size that differs keeps the per-automaton path
    ns2 = ns.copy()
    ns2[-1] = 12
    recs2 = recs.copy()
    recs2[-1, 12] = 0                                      # state 12 of a is past n = 12: cleared
    recs2[-1, 32 + 12] = 0
    recs2[-1, :12] %= 12
    recs2[-1, 32:44] %= 12
    r2 = engine.solve(recs2, ns=ns2)
    assert r2["stats"]["h2d_bytes"] == count * 64 + count
    _check(oracle_mod, recs2, r2, ns=ns2)

"""sbfs_solve_small_noalloc: the solver entry point that allocates nothing.

It exists for callers that cannot allocate device memory -- a plugin inside a
process whose framework already owns the device memory budget, or a loop that
must not let cudaMalloc/cudaFree synchronise the device.  It keeps all of its
working memory in one fixed 16 MiB array inside the library and takes only the
caller's device inputs and outputs.

Here it is called through the C ABI and compared with the regular entry
point: lengths bit-exact, every word replaying to a single state (shortest
words are not unique, so the two paths may return different valid words), the
Cerny check identical.  Each batch is solved twice in a row with the same
inputs: the second call starts from whatever the first left in the shared
array, so identical lengths and violation index show that the call resets
that state.  (The words of the two calls may differ: the pooled kernel
interleaves several automata per warp, so which of several shortest words an
automaton reaches first depends on scheduling; each must replay.)  A batch
with a malformed record (length -2) comes before a clean one, which must not
inherit it.

The file name sorts last so that pytest collects it after every other test:
in a run that stops at the first failure (-x), a failure here cannot keep the
other tests from running.  The tests share no state with other files and pass
alone in a fresh process as well.
"""
import ctypes

import numpy as np
import pytest

import sbfs
from sbfs import problem as P

pytestmark = pytest.mark.gpu


def _call(lib, d_maps, lstride, n, count, d_len, d_words, ws, d_fv):
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    return lib.sbfs_solve_small_noalloc(vp(d_maps), lstride, n, count,
                                        vp(d_len) if d_len is not None else None,
                                        vp(d_words) if d_words is not None else None, ws, vp(d_fv), None)


def _device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    return torch.device("cuda", 0)


def test_noalloc_matches_the_regular_entry_point(oracle_mod):
    import torch
    dev = _device()
    lib = sbfs.load()
    cases = [(60_000, 12, 91), (40_000, 9, 92)]
    with sbfs.Engine(device=0) as eng:
        for count, n, seed in cases:
            recs = P.uniform_maps(count, n, seed)
            recs[3] = P.cerny_record(n)             # the longest case, (n-1)^2 letters
            tight = P.repack(recs, 32, n)
            ws = sbfs.word_stride_for(n)
            d_maps = torch.from_numpy(tight).to(dev)
            ref = eng.solve(tight, n=n, lstride=n)
            runs = []
            for _ in range(2):                      # two calls in a row on the same inputs
                d_len = torch.full((count,), -7, dtype=torch.int32, device=dev)
                d_words = torch.zeros((count, ws), dtype=torch.int64, device=dev)
                d_fv = torch.full((1,), -7, dtype=torch.int64, device=dev)
                torch.cuda.synchronize()
                assert _call(lib, d_maps, n, n, count, d_len, d_words, ws, d_fv) == 0
                torch.cuda.synchronize()
                lens = d_len.cpu().numpy()
                np.testing.assert_array_equal(lens, ref["len"])
                assert lens[3] == (n - 1) ** 2
                words = d_words.cpu().numpy().view(np.uint64)
                assert oracle_mod.replay(tight, lens, words, n=n, lstride=n)[0] == 0
                assert int(d_fv.item()) == ref["first_violation"] == -1
                runs.append((lens, words))
            np.testing.assert_array_equal(runs[0][0], runs[1][0])


def test_noalloc_malformed_record_does_not_leak_into_the_next_call(oracle_mod):
    import torch
    dev = _device()
    lib = sbfs.load()
    n, count = 11, 5000
    recs = P.repack(P.uniform_maps(count, n, 93), 32, n)
    bad = recs.copy()
    bad[17, 4] = n                                  # state index == n: malformed
    ws = sbfs.word_stride_for(n)
    ref = oracle_mod.solve(recs, n=n, lstride=n, words=False)
    for inputs, expect_bad in ((bad, True), (recs, False)):
        d_maps = torch.from_numpy(inputs).to(dev)
        d_len = torch.full((count,), -7, dtype=torch.int32, device=dev)
        d_words = torch.zeros((count, ws), dtype=torch.int64, device=dev)
        d_fv = torch.full((1,), -7, dtype=torch.int64, device=dev)
        assert _call(lib, d_maps, n, n, count, d_len, d_words, ws, d_fv) == 0
        torch.cuda.synchronize()
        lens = d_len.cpu().numpy()
        if expect_bad:
            assert lens[17] == -2
            keep = np.arange(count) != 17
            np.testing.assert_array_equal(lens[keep], ref["len"][keep])
        else:
            np.testing.assert_array_equal(lens, ref["len"])
        assert int(d_fv.item()) == -1


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    dev = _device()
    lib = sbfs.load()
    d_maps = torch.zeros((4, 26), dtype=torch.uint8, device=dev)
    d_len = torch.empty(4, dtype=torch.int32, device=dev)
    d_fv = torch.empty(1, dtype=torch.int64, device=dev)
    assert _call(lib, d_maps, 13, 13, 4, d_len, None, 0, d_fv) == 1   # SBFS_EINVAL
    # lengths are where a malformed record is reported: required
    d_maps12 = torch.zeros((4, 24), dtype=torch.uint8, device=dev)
    assert _call(lib, d_maps12, 12, 12, 4, None, None, 0, d_fv) == 1

"""sbfs_solve_small_noalloc: the solver entry point that allocates nothing.

It exists for callers that cannot allocate device memory -- a plugin inside a
process whose framework already owns the device memory budget, or a loop that
must not let cudaMalloc/cudaFree synchronise the device.  It keeps all of its
working memory in one fixed 16 MiB array inside the library and takes only the
caller's device inputs and outputs.  Here it is called through the C ABI twice
in a row (the second call runs on whatever the first left in that array) and
its lengths, words and Cerny check are compared with the regular entry point's:
lengths bit-exact, every word replaying to a single state (shortest words are
not unique, so the two paths may return different valid words).

This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import sbfs
from sbfs import problem as P

pytestmark = pytest.mark.gpu


def _call(lib, d_maps, lstride, n, count, d_len, d_words, ws, d_fv):
    vp = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    return lib.sbfs_solve_small_noalloc(vp(d_maps), lstride, n, count, vp(d_len),
                                        vp(d_words) if d_words is not None else None, ws, vp(d_fv), None)


def test_noalloc_matches_the_regular_entry_point(oracle_mod):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    lib = sbfs.load()
    cases = [(60_000, 12, 91), (40_000, 9, 92)]
    with sbfs.Engine(device=0) as eng:
        for count, n, seed in cases:
            recs = P.uniform_maps(count, n, seed)
            recs[3] = P.cerny_record(n)             # the longest case, (n-1)^2 letters
            tight = P.repack(recs, 32, n)
            ws = sbfs.word_stride_for(n)
            d_maps = torch.from_numpy(tight).to(dev)
            d_len = torch.full((count,), -7, dtype=torch.int32, device=dev)
            d_words = torch.zeros((count, ws), dtype=torch.int64, device=dev)
            d_fv = torch.full((1,), -7, dtype=torch.int64, device=dev)
            torch.cuda.synchronize()
            assert _call(lib, d_maps, n, n, count, d_len, d_words, ws, d_fv) == 0
            torch.cuda.synchronize()
            ref = eng.solve(tight, n=n, lstride=n)
            lens = d_len.cpu().numpy()
            np.testing.assert_array_equal(lens, ref["len"])
            assert lens[3] == (n - 1) ** 2
            words = d_words.cpu().numpy().view(np.uint64)
            assert oracle_mod.replay(tight, lens, words, n=n, lstride=n)[0] == 0
            assert int(d_fv.item()) == ref["first_violation"] == -1


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = sbfs.load()
    dev = torch.device("cuda", 0)
    d_maps = torch.zeros((4, 26), dtype=torch.uint8, device=dev)
    d_len = torch.empty(4, dtype=torch.int32, device=dev)
    d_fv = torch.empty(1, dtype=torch.int64, device=dev)
    assert _call(lib, d_maps, 13, 13, 4, d_len, None, 0, d_fv) == 1   # SBFS_EINVAL

"""The C-ABI library loads and exports every symbol include/*.h declares.
No compute calls here: these run without a GPU."""
import ctypes
import glob
import os
import re

import pytest

import sbfs
from sbfs import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"SBFS_API\s+[^;(]*?\b(sbfs_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_is_built():
    assert os.path.exists(_native.LIB_PATH), "run __graft_entry__.build()"


def test_every_declared_symbol_is_exported():
    lib = _native.load()
    names = declared_symbols()
    assert len(names) >= 10
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_list_covers_header():
    assert declared_symbols() <= set(sbfs.EXPORTS)


def test_pure_helpers():
    lib = _native.load()
    assert lib.sbfs_abi_version() == 2
    assert lib.sbfs_word_stride(12) == 2      # 121 bits
    assert lib.sbfs_word_stride(28) == 12     # 729 bits
    assert lib.sbfs_word_stride(2) == 1
    assert lib.sbfs_status_string(1) == b"invalid argument"
    cfg = _native.Config()
    assert lib.sbfs_config_default(ctypes.byref(cfg)) == 0
    assert cfg.device == -1 and cfg.slack == 0


def test_null_arguments_are_rejected_without_a_device():
    lib = _native.load()
    assert lib.sbfs_config_default(None) == 1
    assert lib.sbfs_destroy(None) == 0
    assert lib.sbfs_create(None, None) == 1
    fv = ctypes.c_int64()
    st = lib.sbfs_solve_batch(None, None, 32, None, 8, 0, None, None, 0, ctypes.byref(fv), None)
    assert st == 1


def test_server_entry_points_reject_null_handles():
    lib = _native.load()
    assert lib.sbfs_server_config_default(None) == 1
    assert lib.sbfs_server_start(None, None) == 1
    rid = ctypes.c_uint64()
    a = (ctypes.c_uint8 * 3)(1, 2, 0)
    assert lib.sbfs_server_submit(None, a, a, 3, ctypes.byref(rid)) == 1
    ids = (ctypes.c_uint64 * 1)()
    ns = (ctypes.c_uint8 * 1)(3)
    recs = (ctypes.c_uint8 * 64)()
    assert lib.sbfs_server_submit_many(None, recs, 32, ns, 1, ids) == 1
    got = ctypes.c_int32()
    assert lib.sbfs_server_poll(None, None, 0, ctypes.byref(got), 0) == 1
    assert lib.sbfs_server_cancel(None, 7) == 1
    assert lib.sbfs_server_stats_get(None, None) == 1
    assert lib.sbfs_server_reset_peak(None) == 1
    assert lib.sbfs_server_stop(None) == 0


def test_noalloc_entry_rejects_bad_sizes_before_touching_a_device():
    """The allocation-free entry point serves n <= 12 only (its fixed scratch is
    sized for that) and checks its arguments before any CUDA call."""
    lib = _native.load()
    fv = ctypes.c_int64()
    maps = (ctypes.c_uint8 * 64)()
    for n, lstride, count in [(0, 32, 1), (13, 32, 1), (20, 32, 1), (8, 4, 1), (8, 33, 1), (8, 32, -1)]:
        assert lib.sbfs_solve_small_noalloc(maps, lstride, n, count, None, None, 0, ctypes.byref(fv), None) == 1
    assert lib.sbfs_solve_small_noalloc(maps, 32, 8, 1, None, None, 0, None, None) == 1   # no violation slot
    assert lib.sbfs_solve_small_noalloc(None, 32, 8, 1, None, None, 0, ctypes.byref(fv), None) == 1
    words = (ctypes.c_uint64 * 2)()
    assert lib.sbfs_solve_small_noalloc(maps, 32, 8, 1, None, words, 0, ctypes.byref(fv), None) == 1
    # lengths are required: a malformed record is reported only through them
    assert lib.sbfs_solve_small_noalloc(maps, 32, 8, 1, None, words, 2, ctypes.byref(fv), None) == 1

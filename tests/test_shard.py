"""Multi-rank sharding logic (sbfs/shard.py) on CPU: two gloo ranks, each
solving its contiguous range with the CPU oracle as a stand-in solver, results
gathered to rank 0 and compared with one process solving everything.  Also a
planted violation (the oracle's slack) must come back with its global index."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sbfs import problem as P
from sbfs.shard import shard_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_path):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    for p in (os.path.join(root, "gpgpu-binary-automaton-synchronizing-algorithms_b200"),
              os.path.join(root, "oracle")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    import oracle
    from sbfs import problem as P
    from sbfs.shard import solve_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ns = P.uniform_sizes(3001, 4, 14, 5)
    recs = P.uniform_maps(3001, ns, 6)
    recs[2500] = P.cerny_record(int(ns[2500]))

    def cpu_solve(r, ns=None, n=0, lstride=32, word_stride=1):
        return oracle.solve(r, ns=ns, n=n, lstride=lstride, word_stride=word_stride, slack=1)

    lens, words, fv = solve_sharded(cpu_solve, recs, ns, 0, 32, 3)
    if rank == 0:
        np.savez(out_path, lens=lens, words=words, fv=fv)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_range_partition():
    for count in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(count, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == count
            for (b0, e0), (b1, e1) in zip(spans, spans[1:]):
                assert e0 == b1 and b0 <= e0


def test_two_gloo_ranks_match_one_process(tmp_path, oracle_mod):
    out = str(tmp_path / "gathered.npz")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    g = np.load(out)
    ns = P.uniform_sizes(3001, 4, 14, 5)
    recs = P.uniform_maps(3001, ns, 6)
    recs[2500] = P.cerny_record(int(ns[2500]))
    ref = oracle_mod.solve(recs, ns=ns, word_stride=3, slack=1)
    np.testing.assert_array_equal(g["lens"], ref["len"])
    assert oracle_mod.replay(recs, g["lens"], g["words"], ns=ns)[0] == 0
    assert int(g["fv"]) == ref["first_violation"] >= 0   # planted via slack, global index

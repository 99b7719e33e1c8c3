"""Multi-GPU sharding of a batch: one process per GPU, contiguous automaton
ranges, no exchange on the data path.

Automata are independent, so the batch splits into contiguous ranges per rank,
as the reference splits it per stream (GPGPU/GPU/SlimGPUQueue.cs:74,100-101)
and per CPU thread (GPGPU/CPU/SlimCPUUntweaked.cs:33-47).  Each rank solves its
own range on its own GPU; the only collectives are control: gathering the
per-rank lengths/words to one rank and reducing the first Cerny violation
(minimum global index).  The solver is a parameter so the same logic runs with
the CUDA engine on GPUs or, in tests, with any CPU callable under gloo.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import numpy as np


def shard_range(count: int, world: int, rank: int) -> Tuple[int, int]:
    """Contiguous [begin, end) of rank `rank` out of `world` (ceil partition)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    part = (count + world - 1) // world
    begin = min(rank * part, count)
    return begin, min(begin + part, count)


def solve_sharded(solve: Callable[..., dict], recs: np.ndarray, ns: Optional[np.ndarray], n: int,
                  lstride: int, word_stride: int, group=None, dst: int = 0):
    """Solve this rank's range with `solve(recs, ns=..., n=..., lstride=...,
    word_stride=...)` and gather everything to rank `dst`.

    Returns (len, words, first_violation) on `dst` (global arrays, global
    index) and (None, None, first_violation) elsewhere.  The first violation is
    reduced on every rank.
    """
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    count = recs.shape[0]
    b, e = shard_range(count, world, rank)
    part = (count + world - 1) // world
    local = solve(recs[b:e], ns=None if ns is None else ns[b:e], n=n, lstride=lstride, word_stride=word_stride)
    lens = np.full(part, -3, dtype=np.int32)
    words = np.zeros((part, word_stride), dtype=np.uint64)
    lens[: e - b] = local["len"]
    if local.get("words") is not None:
        words[: e - b] = local["words"]
    fv = local.get("first_violation", -1)
    fv_global = b + fv if fv >= 0 else np.iinfo(np.int64).max
    t_fv = torch.tensor([fv_global], dtype=torch.int64)
    t_len = torch.from_numpy(lens)
    t_words = torch.from_numpy(words.view(np.int64))
    backend = dist.get_backend(group)
    if backend == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
        t_fv, t_len, t_words = t_fv.to(dev), t_len.to(dev), t_words.to(dev)
    dist.all_reduce(t_fv, op=dist.ReduceOp.MIN, group=group)
    gl = [torch.empty_like(t_len) for _ in range(world)] if rank == dst else None
    gw = [torch.empty_like(t_words) for _ in range(world)] if rank == dst else None
    if backend == "nccl":
        # NCCL has no gather; all_gather keeps every rank in the same collective
        gl = [torch.empty_like(t_len) for _ in range(world)]
        gw = [torch.empty_like(t_words) for _ in range(world)]
        dist.all_gather(gl, t_len, group=group)
        dist.all_gather(gw, t_words, group=group)
    else:
        dist.gather(t_len, gl, dst=dst, group=group)
        dist.gather(t_words, gw, dst=dst, group=group)
    first = int(t_fv.item())
    first = -1 if first == np.iinfo(np.int64).max else first
    if rank != dst:
        return None, None, first
    all_len = torch.cat([x.cpu() for x in gl]).numpy()[:count]
    all_words = torch.cat([x.cpu() for x in gw]).numpy().view(np.uint64)[:count]
    return all_len, all_words, first

"""bench.py -- throughput of exact shortest-synchronizing-word search on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sbfs|reference]
                    [--workload n12|n8|mixed|large]

Default workload (the benchmark's headline configuration): 1,000,000 uniform
random binary automata with n = 12 states per GPU, tight 24-byte records,
seeded synthetic inputs.  By default the n12 and n8 batches are the
reference's own: Problem.FillArrayOfProblems with .NET System.Random and the
benchmark's seed 1234567 + count (rank r > 0 adds 7919 * r); --inputs hash
draws them from a counter hash instead.  One step = one pass of the power-set BFS over the
whole batch, producing every shortest length (or the non-synchronizing flag)
and one shortest word per automaton.

  value    automata/s over all ranks with records already resident in HBM
           (sbfs_solve_batch_device), CUDA events on the launching stream, L2
           flushed (256 MiB write) before every timed step, max over ranks.
  e2e      the same metric through sbfs_solve_batch with pinned host buffers:
           host->device copy of the records and device->host copy of lengths
           and words inside every timed step.
  roofline the BFS kernel against HBM (algorithmic I/O bytes) and, under
           "onchip", against shared-memory bandwidth (28 B per expansion).
  cpu_baseline  the CPU restatement of the reference's timed solver
           (SlimCPU4bits13, Verify mode) on this host's cores, rank 0, N = 1.

With --impl reference the same workload runs through that CPU restatement
only, on all host threads (the reference itself is C#/.NET and cannot run
here).  Multi-GPU: one process per GPU (torchrun); every rank solves its own
1M-automaton shard (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import signal
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gpgpu-binary-automaton-synchronizing-algorithms_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "exact automata/s (n=12 batch) and p50/p99 latency, batched vs plain on 1 B200"
UNIT = "automata/s"
SMEM_BYTES_PER_EXPANSION = 28     # 4 pop + 2 x (4 + 4) bitmap word RMW + 2 x 4 push
# level slots (n >= 21): bitmaps and frontiers live in HBM, so the search itself
# is HBM traffic: 4 E frontier reads + 8 E bitmap-word probes + 4 D bitmap writes
# + 4 D frontier writes, with D (discoveries) = E (expansions) over a whole search
LEVEL_BYTES_PER_EXPANSION = 20
FLUSH_BYTES = 256 << 20           # > 126 MB L2


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["sbfs", "reference"], default="sbfs")
    ap.add_argument("--workload", choices=["n12", "n8", "mixed", "large", "serving"], default="n12")
    ap.add_argument("--rates", default="2000,8000,32000,128000,0",
                    help="serving: offered request rates per second (0 = submit all at once)")
    ap.add_argument("--count", type=int, default=0, help="automata per GPU (0 = the workload's size)")
    ap.add_argument("--max-batch", type=int, default=0, help="serving: small requests per mini-batch (0 = 8192)")
    ap.add_argument("--max-levels", type=int, default=0, help="serving: levels per launch batch (0 = 16)")
    ap.add_argument("--inputs", choices=["reference", "hash"], default="reference",
                    help="n12/n8: the reference's System.Random batch or a counter-hash batch")
    ap.add_argument("--cpu-seconds", type=float, default=1.5, help="wall time of the CPU baseline sample")
    ap.add_argument("--plain-sample", type=int, default=2000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="n12: skip the serving-latency summary")
    ap.add_argument("--no-tune", action="store_true", help="keep the default kernel shapes")
    ap.add_argument("--no-graph", action="store_true", help="launch every step directly, no CUDA graphs")
    ap.add_argument("--chunk", type=int, default=0, help="host path: automata per chunk (0 = library default)")
    ap.add_argument("--streams", type=int, default=0, help="host path: chunks in flight (0 = library default)")
    ap.add_argument("--large-n", default="24,26,28", help="large workload: the state counts to include")
    ap.add_argument("--large-kinds", default="random,cerny,perm",
                    help="large workload: which families to include (random, cerny, perm)")
    ap.add_argument("--level-arena-mb", type=int, default=0, help="HBM budget of the n > 20 level slots")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def _uniform_batch(count: int, n: int, rank: int, inputs: str, hash_seed: int):
    from sbfs import dotnet_random as D
    from sbfs import problem as P
    if inputs == "reference":
        seed = D.BENCHMARK_SEED + count + 7919 * rank
        return D.fill_array_of_problems(count, n, seed, lstride=n), f"System.Random, seed {seed}"
    return P.repack(P.uniform_maps(count, n, hash_seed + 1000 * rank), 32, n), f"counter hash 0x{hash_seed:X}"


def make_workload(name: str, count: int, rank: int, large_n=(24, 26, 28), kinds=("random", "cerny", "perm"),
                  inputs: str = "reference"):
    import numpy as np
    from sbfs import problem as P

    seed_base = 0x5EED
    if name == "n12":
        count = count or 1_000_000
        recs, seed = _uniform_batch(count, 12, rank, inputs, seed_base + 1)
        return dict(recs=recs, ns=None, n=12, lstride=12, max_n=12, count=count, seed=seed,
                    desc=f"batched uniform: {count:,} random binary automata, n=12, lengths + shortest words")
    if name == "n8":
        count = count or 10_000
        recs, seed = _uniform_batch(count, 8, rank, inputs, seed_base + 0)
        return dict(recs=recs, ns=None, n=8, lstride=8, max_n=8, count=count, seed=seed,
                    desc=f"plain config: {count:,} random binary automata, n=8")
    if name == "mixed":
        count = count or 200_000
        ns = P.uniform_sizes(count, 6, 20, seed_base + 2 + 1000 * rank)
        recs = P.uniform_maps(count, ns, seed_base + 2 + 1000 * rank)
        for i in range(0, count, 100):   # 1% Cerny family
            recs[i] = P.cerny_record(int(ns[i]))
        return dict(recs=recs, ns=ns, n=0, lstride=32, max_n=20, count=count, seed="counter hash 0x5EED",
                    desc=f"batched mixed: {count:,} automata, n uniform in 6..20, 1% Cerny family")
    if name == "large":
        rows, ns = [], []
        for n in large_n:
            if "random" in kinds:
                r = P.uniform_maps(64, n, seed_base + 4 + n)
                rows.extend(list(r))
                ns.extend([n] * 64)
            if "cerny" in kinds:
                rows.append(P.cerny_record(n)); ns.append(n)
            if "perm" in kinds:
                rows.append(P.perm_merge_record(n, seed_base + 5 + n)); ns.append(n)
        recs = np.stack(rows)
        ns = np.array(ns, dtype=np.uint8)
        return dict(recs=recs, ns=ns, n=0, lstride=32, max_n=max(large_n), count=len(ns),
                    seed="counter hash 0x5EED", desc=f"large single instances: n={','.join(map(str, large_n))} x "
                         f"({' + '.join(kinds)})")
    raise ValueError(name)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.lines = []
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.send_signal(signal.SIGTERM)
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU legs (oracle restatement of the reference's CPU solver)
# ---------------------------------------------------------------------------

def cpu_throughput(wl, seconds: float, threads: int):
    """SlimCPU4bits13 restatement (n <= 16) or SlimCPUUntweaked (otherwise) over
    passes of the workload's records until `seconds` of wall time."""
    import numpy as np
    import oracle

    recs, n = wl["recs"], wl["n"]
    t0 = time.perf_counter()
    done, passes = 0, 0
    while True:
        if wl["ns"] is None and n <= 16:
            oracle.verify4(recs, n=n, lstride=wl["lstride"], threads=threads)
        else:
            oracle.solve(recs, ns=wl["ns"], n=n, lstride=wl["lstride"], words=False, threads=threads)
        done += recs.shape[0]
        passes += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    kind = "SlimCPU4bits13 (nibble table, Verify mode)" if (wl["ns"] is None and n <= 16) else \
        "SlimCPUUntweaked (lengths)"
    return done / dt, dt, passes, kind


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    wl = make_workload(args.workload, args.count, 0, tuple(int(x) for x in args.large_n.split(",")),
                       tuple(args.large_kinds.split(",")), args.inputs)
    threads = os.cpu_count() or 1
    import oracle

    oracle.build()
    for _ in range(max(args.warmup, 0)):
        cpu_throughput(wl, 0.0, threads)
    step_ms = []
    for _ in range(args.steps):
        rate, dt, passes, kind = cpu_throughput(wl, 0.0, threads)
        step_ms.append(dt * 1e3)
    ms = statistics.mean(step_ms)
    value = wl["count"] / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic", "impl": "reference",
        "config": {"workload": wl["desc"], "automata": wl["count"], "n": wl["n"] or "6..28", "seed": wl["seed"]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} passes over the full {wl['count']:,}-automaton batch "
                                   f"({kind}, C restatement; the C# reference cannot run here)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def load_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary of this kernel, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(path))
    except (OSError, ValueError):
        return None
    ent = d.get(kernel)
    return ent.get("dram_bytes_per_launch") if isinstance(ent, dict) else None


def run_sbfs(args):
    import numpy as np
    import torch

    import sbfs

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    wl = make_workload(args.workload, args.count, rank, tuple(int(x) for x in args.large_n.split(",")),
                       tuple(args.large_kinds.split(",")), args.inputs)
    count, lstride = wl["count"], wl["lstride"]
    ws = sbfs.word_stride_for(wl["max_n"])
    import tempfile
    tune_cache = os.path.join(tempfile.gettempdir(), "sbfs_tune_cache.txt")
    eng = sbfs.Engine(device=dev.index, autotune=not args.no_tune, tune_cache=tune_cache,
                      use_graph=not args.no_graph, level_arena_bytes=args.level_arena_mb << 20,
                      chunk=args.chunk, streams=args.streams)
    plan = eng.plan()   # runs the autotuner (or reads its cache) before any timing

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident leg ------------------------------------------------
    # a dedicated stream: the events, the L2 flush and the library's kernels all
    # go on it (the legacy default stream would hand the library a NULL stream)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    d_maps = torch.from_numpy(wl["recs"]).to(dev)
    d_ns = torch.from_numpy(wl["ns"]).to(dev) if wl["ns"] is not None else None
    d_len = torch.empty(count, dtype=torch.int32, device=dev)
    d_words = torch.empty((count, ws), dtype=torch.int64, device=dev)
    d_fv = torch.empty(1, dtype=torch.int64, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def step_device():
        eng.solve_device(d_maps, lstride, count, n=wl["n"], d_ns=d_ns, max_n=wl["max_n"], d_len=d_len,
                         d_words=d_words, word_stride=ws, d_first_violation=d_fv, stream=stream)

    for i in range(args.warmup):
        flush.fill_(i)
        step_device()
        eng.wait_device()
    visible = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip().isdigit()]
    gpu_index = int(visible[dev.index]) if dev.index < len(visible) else dev.index
    clocks = ClockSampler(gpu_index) if rank == 0 else None
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(i + 1)                 # untimed: evicts the records from L2
        evs[i][0].record(stream)
        step_device()
        evs[i][1].record(stream)
    barrier()
    stats = eng.wait_device()
    clk = clocks.stop() if clocks else None
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = statistics.mean(step_ms)
    ms_max = max_over_ranks(ms)
    value = count * world / (ms_max / 1e3)
    launches_per_step = int(stats.get("launches", 0))
    expanded_per_step = int(stats.get("expanded", 0))
    fv = int(d_fv.item())
    lens = d_len.cpu().numpy()
    sync_frac = float((lens >= 0).mean()) if count else 0.0

    # ---- end-to-end leg through the host API ----------------------------------
    e2e = None
    if not args.no_e2e:
        h_maps = torch.from_numpy(wl["recs"]).pin_memory()
        h_ns = torch.from_numpy(wl["ns"]).pin_memory() if wl["ns"] is not None else None
        h_len = torch.empty(count, dtype=torch.int32).pin_memory()
        h_words = torch.empty((count, ws), dtype=torch.int64).pin_memory()
        out = (h_len.numpy(), h_words.numpy().view(np.uint64))
        for i in range(args.warmup):
            eng.solve(h_maps.numpy(), ns=None if h_ns is None else h_ns.numpy(), n=wl["n"], lstride=lstride,
                      word_stride=ws, out=out)
        e2e_ms = []
        barrier()
        for i in range(args.steps):
            flush.fill_(i + 7)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = eng.solve(h_maps.numpy(), ns=None if h_ns is None else h_ns.numpy(), n=wl["n"],
                          lstride=lstride, word_stride=ws, out=out)
            e2e_ms.append((time.perf_counter() - t0) * 1e3)
        barrier()
        e2e_mean = max_over_ranks(statistics.mean(e2e_ms))
        st = r["stats"]
        e2e = {"value": count * world / (e2e_mean / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(st["h2d_bytes"]), "d2h_bytes_per_step": int(st["d2h_bytes"]) + 0,
               "ms_per_step": e2e_mean,
               "latency_ms": {"p50": statistics.median(e2e_ms),
                              "p99": sorted(e2e_ms)[min(len(e2e_ms) - 1, int(0.99 * len(e2e_ms)))]}}
        if not np.array_equal(r["len"], lens):
            raise SystemExit("host and device paths disagree")

    # ---- plain form (one automaton per launch) on a sample ------------------
    plain = None
    if rank == 0 and args.plain_sample > 0:
        k = min(args.plain_sample, count)
        sub = wl["recs"][:k]
        ns_sub = wl["ns"][:k] if wl["ns"] is not None else None
        eng.solve(sub[: min(k, 50)], ns=None if ns_sub is None else ns_sub[:50], n=wl["n"], lstride=lstride,
                  plain=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rp = eng.solve(sub, ns=ns_sub, n=wl["n"], lstride=lstride, plain=True)
        dt = time.perf_counter() - t0
        if not np.array_equal(rp["len"], lens[:k]):
            raise SystemExit("plain and batched forms disagree")
        plain = {"value": k / dt, "unit": UNIT, "sample": k, "kernel_ms": rp["stats"]["kernel_ms"],
                 "batched_over_plain": value / world / (k / dt)}

    # ---- CPU baseline (rank 0, N = 1) --------------------------------------
    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        rate, dt, passes, kind = cpu_throughput(wl, args.cpu_seconds, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{passes} passes over the same {count:,}-automaton batch in {dt:.2f} s wall "
                         f"({kind}; C restatement, the C# reference cannot run here)"}

    if rank == 0:
        # p50/p99 of the metric's serving half: single-automaton requests through the
        # serving loop (n log-uniform 8..24, 5 % Cerny), at 32K requests/s and all at once
        serving = None
        if args.workload == "n12" and not args.no_serving:
            def brief(e):
                return {"offered_per_s": e["offered_per_s"], "achieved_per_s": e["achieved_automata_per_s"],
                        "p50_ms_n_le_20": e["latency_ms_n_le_20"]["p50"],
                        "p99_ms_n_le_20": e["latency_ms_n_le_20"]["p99"],
                        "p99_ms_all": e["latency_ms"]["p99"]}
            serving = {"requests": 10_000, "sweep": [brief(e) for e in serve_sweep(10_000, [32000.0, 0.0])],
                       "full_sweep": "bench.py --workload serving"}
        # roofline of the dominant kernel (the step is one BFS launch plus tiny bookkeeping)
        kern = [c["kernel"] for c in plan.get("classes", []) if c["max_n"] >= wl["max_n"]][:1]
        kernel = kern[0] if kern else "k_pool"
        rec_bytes = 2 * lstride + (1 if wl["ns"] is not None else 0)
        alg_bytes = count * (rec_bytes + 4 + 8 * ws)
        if kernel == "k_level":
            alg_bytes += expanded_per_step * LEVEL_BYTES_PER_EXPANSION
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        achieved = alg_bytes / (ms / 1e3) / 1e9
        sm_clock_ghz = (clk or {}).get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        smem_peak = 148 * 128 * (sm_clock_ghz / 1e3)   # GB/s at the measured SM clock
        onchip = expanded_per_step * SMEM_BYTES_PER_EXPANSION / (ms / 1e3) / 1e9
        traffic = load_traffic(kernel)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": {"workload": wl["desc"], "automata_per_gpu": count, "n": wl["n"] or "mixed",
                       "record_bytes": rec_bytes, "word_stride_u64": ws, "kernel": kernel,
                       "l2": "flushed by a 256 MiB write before every timed step",
                       "parallelism": f"{world} GPU(s), automata sharded by rank, no collective on the data path",
                       "seed": wl["seed"]},
            "e2e": e2e,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic,
                         "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "algorithmic_bytes": ("records + results" if kernel != "k_level" else
                                               f"records + results + {LEVEL_BYTES_PER_EXPANSION} B per expansion "
                                               "(HBM bitmaps and queues)"),
                         "onchip": {"bound": "smem", "achieved": onchip, "peak": smem_peak, "unit": "GB/s",
                                    "frac": onchip / smem_peak,
                                    "bytes_per_expansion": SMEM_BYTES_PER_EXPANSION,
                                    "expansions_per_launch": expanded_per_step,
                                    "peak_source": "nominal 148 SM x 128 B/clk at the sampled SM clock"}},
            "cpu_baseline": cpu,
            "plain": plain,
            "clocks": clk,
            "gpu_launches": launches_per_step * args.steps,
            "latency_ms": {"p50": statistics.median(step_ms),
                           "p99": sorted(step_ms)[min(len(step_ms) - 1, int(0.99 * len(step_ms)))]},
            "results": {"synchronizing_fraction": sync_frac, "first_violation": fv,
                        "max_length": int(lens.max()) if count else 0},
            "plan": plan,
        }
        if serving:
            line["serving"] = serving
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# serving: open-loop Poisson arrivals of single-automaton requests
# ---------------------------------------------------------------------------

def serve_sweep(count, rates, max_batch=0, max_levels=0):
    """Open-loop Poisson sweep of single-automaton requests through the serving
    loop (n log-uniform 8..24, 5 % Cerny family); one entry per offered rate
    (0 = all submitted at once)."""
    import threading

    import numpy as np

    from sbfs import problem as P
    from sbfs.server import Server

    seed = 0x5EED + 3
    ns = P.log_uniform_sizes(count, 8, 24, seed)
    recs = P.uniform_maps(count, ns, seed + 1)
    cerny = np.arange(0, count, 20)          # 5% Cerny family
    for i in cerny:
        recs[i] = P.cerny_record(int(ns[i]))
    a_rows = [np.ascontiguousarray(recs[i, :ns[i]]) for i in range(count)]
    b_rows = [np.ascontiguousarray(recs[i, 32:32 + ns[i]]) for i in range(count)]
    rng = np.random.default_rng(seed)
    sweep = []
    srv = Server(device=0, max_batch=max_batch, max_levels=max_levels)
    # warm-up: the whole request set once, so every kernel the sweep uses has been
    # loaded and launched before anything is timed
    warm = [srv.submit(a_rows[i], b_rows[i], int(ns[i])) for i in range(count)]
    srv.wait_all(warm)
    for rate in rates:
        srv.reset_peak()
        gaps = rng.exponential(1.0 / rate, count) if rate > 0 else np.zeros(count)
        times = np.cumsum(gaps)
        ids = [0] * count
        refused = [0]

        def submitter():
            t0 = time.perf_counter()
            for i in range(count):
                target = t0 + times[i]
                while True:
                    now = time.perf_counter()
                    if now >= target:
                        break
                    if target - now > 2e-4:
                        time.sleep((target - now) * 0.5)
                while True:
                    try:
                        ids[i] = srv.submit(a_rows[i], b_rows[i], int(ns[i]))
                        break
                    except Exception:
                        refused[0] += 1
                        time.sleep(1e-4)

        th = threading.Thread(target=submitter)
        t_start = time.perf_counter()
        th.start()
        results = {}
        while len(results) < count:
            for r in srv.poll(timeout_ms=20):
                results[r["id"]] = r
            if not th.is_alive() and len(results) < count and time.perf_counter() - t_start > 600:
                raise SystemExit("serving run did not finish")
        th.join()
        wall = time.perf_counter() - t_start
        st = srv.stats()
        by_id = [results[i] for i in ids]
        lat = np.array([r["done_ms"] - r["submit_ms"] for r in by_id])
        small = np.array([int(r["n"]) <= 20 for r in by_id])
        tiny = np.array([int(r["n"]) <= 16 for r in by_id])
        mid = small & ~tiny
        first = min(r["submit_ms"] for r in by_id)
        last = max(r["done_ms"] for r in by_id)
        entry = {
            "offered_per_s": rate if rate > 0 else "all at once",
            "achieved_automata_per_s": count / ((last - first) / 1e3),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "latency_ms_n_le_20": {"p50": float(np.percentile(lat[small], 50)),
                                   "p99": float(np.percentile(lat[small], 99))},
            "latency_ms_n_le_16": {"p50": float(np.percentile(lat[tiny], 50)),
                                   "p99": float(np.percentile(lat[tiny], 99))},
            "latency_ms_n_17_20": {"p50": float(np.percentile(lat[mid], 50)),
                                   "p99": float(np.percentile(lat[mid], 99))},
            "peak_arena_bytes": int(st["arena_peak"]), "submit_retries": refused[0], "wall_s": wall,
        }
        sweep.append(entry)
        print(json.dumps({"serving_rate": entry}), file=sys.stderr, flush=True)
    srv.stop()
    return sweep


def run_serving(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    count = args.count or 20_000
    rates = [float(r) for r in args.rates.split(",")]
    sweep = serve_sweep(count, rates, args.max_batch, args.max_levels)
    best = max(sweep, key=lambda e: e["achieved_automata_per_s"])
    line = {
        "metric": METRIC, "value": best["achieved_automata_per_s"], "unit": UNIT, "n_gpus": 1, "steps": len(rates),
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u16", "data": "synthetic",
        "config": {"workload": f"serving: {count:,} single-automaton requests, n log-uniform 8..24, 5% Cerny, "
                               "open-loop Poisson arrivals at swept rates", "rates": args.rates},
        "serving": sweep,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    return run_sbfs(args)


if __name__ == "__main__":
    sys.exit(main())

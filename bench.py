"""bench.py -- throughput of exact shortest-synchronizing-word search on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sbfs|reference]
                    [--workload n12|n8|n13|mixed|large|serving]

Default workload (the benchmark's headline configuration): 1,000,000 uniform
random binary automata with n = 12 states per GPU, tight 24-byte records,
seeded synthetic inputs.  By default the n12, n8 and n13 batches are the
reference's own: Problem.FillArrayOfProblems with .NET System.Random and the
benchmark's seed 1234567 + count (rank r > 0 adds 7919 * r); --inputs hash
draws them from a counter hash instead.  One step = one pass of the power-set
BFS over the whole batch, producing every shortest length (or the
non-synchronizing flag) and one shortest word per automaton.

  value    automata/s over all ranks with records already resident in HBM
           (sbfs_solve_batch_device), CUDA events on the launching stream, L2
           flushed (256 MiB write) before every timed step, max over ranks.
  e2e      the same metric through sbfs_solve_batch with pinned host buffers:
           host->device copy of the records and device->host copy of lengths
           and words inside every timed step.
  roofline the dominant BFS kernel.  On-chip workloads (n <= 20): 28 B of
           shared-memory traffic per expansion against the SM's shared-memory
           bandwidth; the level slots (n >= 21): 20 B of HBM search traffic
           per expansion against measured HBM bandwidth.
  cpu_baseline  the CPU restatement of the reference's timed solver
           (SlimCPU4bits13, Verify mode) on this host's cores, rank 0, N = 1.
  mixed, large, n13  summaries of the other configurations, each timed on the
           device with its own CPU restatement beside it (N = 1 only).

With --impl reference the same workload runs through that CPU restatement
only, on all host threads (the reference itself is C#/.NET and cannot run
here); its batch is generated by the restatement's own System.Random, so that
arm never loads the CUDA library.  Multi-GPU: one process per GPU; every rank
solves its own 1M-automaton shard (weak scaling, no data-path collective).
`--gpus N` outside torchrun starts the N ranks itself.
"""
from __future__ import annotations

import argparse
import json
import os
import signal
import socket
import statistics
import subprocess
import sys
import threading
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
L2_NOTE = "flushed by a 256 MiB device write before every timed GPU step"
NOMINAL_SMEM_BYTES_PER_CLK = 128  # 32 banks x 4 B per SM per clock
# the reference's published n = 13 numbers (median automata/s, batch 2^21)
PUBLISHED_N13 = {"SlimGPUQueue (GTX 1060)": 1953926, "SlimCPU (Ryzen 7, 16 threads)": 2281843,
                 "source": "Cerny conjecture verification algorithms.pdf p.18, Median row"}


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["sbfs", "reference"], default="sbfs")
    ap.add_argument("--workload", choices=["n12", "n8", "n13", "mixed", "large", "serving"], default="n12")
    ap.add_argument("--rates", default="2000,8000,32000,128000,512000,0",
                    help="serving: offered request rates per second (0 = submit all at once)")
    ap.add_argument("--count", type=int, default=0, help="automata per GPU (0 = the workload's size)")
    ap.add_argument("--max-batch", type=int, default=0, help="serving: small requests per mini-batch (0 = 8192)")
    ap.add_argument("--max-levels", type=int, default=0, help="serving: levels per launch batch (0 = 16)")
    ap.add_argument("--inputs", choices=["reference", "hash"], default="reference",
                    help="n12/n8/n13: the reference's System.Random batch or a counter-hash batch")
    ap.add_argument("--cpu-seconds", type=float, default=1.5, help="wall time of the CPU baseline sample")
    ap.add_argument("--plain-sample", type=int, default=2000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-serving", action="store_true", help="n12: skip the serving-latency summary")
    ap.add_argument("--serving-requests", type=int, default=100_000,
                    help="n12: requests of each rate of the serving-latency summary")
    ap.add_argument("--no-extra", action="store_true", help="n12: skip the mixed / large / n13 summaries")
    ap.add_argument("--extra-steps", type=int, default=5, help="timed steps of each extra summary")
    ap.add_argument("--no-tune", action="store_true", help="keep the default kernel shapes")
    ap.add_argument("--no-graph", action="store_true", help="launch every step directly, no CUDA graphs")
    ap.add_argument("--chunk", type=int, default=0, help="host path: automata per chunk (0 = library default)")
    ap.add_argument("--streams", type=int, default=0, help="host path: chunks in flight (0 = library default)")
    ap.add_argument("--large-n", default="24,26,28", help="large workload: the state counts to include")
    ap.add_argument("--large-kinds", default="random,cerny,perm",
                    help="large workload: which families to include (random, cerny, perm)")
    ap.add_argument("--level-arena-mb", type=int, default=0, help="HBM budget of the n > 20 level slots")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------

def _reference_batch(count: int, n: int, seed: int, lstride: int, gen: str):
    """Problem.FillArrayOfProblems(count, n, seed): from the product library's
    generator (gen = "sbfs") or from the CPU restatement's (gen = "oracle",
    the reference arm, which must not load the CUDA library)."""
    if gen == "oracle":
        import oracle
        return oracle.fill_array_of_problems(count, n, seed, lstride, threads=os.cpu_count() or 1)
    from sbfs import dotnet_random as D
    return D.fill_array_of_problems(count, n, seed, lstride=lstride)


def _uniform_batch(count: int, n: int, rank: int, inputs: str, hash_seed: int, gen: str):
    from sbfs import problem as P
    if inputs == "reference":
        seed = 1234567 + count + 7919 * rank      # GPGPU/Program.cs:94
        return _reference_batch(count, n, seed, n, gen), f"System.Random, seed {seed}"
    return P.repack(P.uniform_maps(count, n, hash_seed + 1000 * rank), 32, n), f"counter hash 0x{hash_seed:X}"


def make_workload(name: str, count: int = 0, rank: int = 0, large_n=(24, 26, 28),
                  kinds=("random", "cerny", "perm"), inputs: str = "reference", gen: str = "sbfs"):
    import numpy as np
    from sbfs import problem as P

    seed_base = 0x5EED
    if name in ("n12", "n8", "n13"):
        n = int(name[1:])
        count = count or {12: 1_000_000, 8: 10_000, 13: 1 << 21}[n]
        recs, seed = _uniform_batch(count, n, rank, inputs, seed_base + {8: 0, 12: 1, 13: 6}[n], gen)
        desc = {12: f"batched uniform: {count:,} random binary automata, n=12, lengths + shortest words",
                8: f"plain config: {count:,} random binary automata, n=8",
                13: f"published-number point: {count:,} random binary automata, n=13 (Program.cs batch)"}[n]
        return dict(name=name, recs=recs, ns=None, n=n, lstride=n, max_n=n, count=count, seed=seed, desc=desc)
    if name == "mixed":
        count = count or 200_000
        ns = P.uniform_sizes(count, 6, 20, seed_base + 2 + 1000 * rank)
        recs = P.uniform_maps(count, ns, seed_base + 2 + 1000 * rank)
        for i in range(0, count, 100):   # 1% Cerny family
            recs[i] = P.cerny_record(int(ns[i]))
        return dict(name=name, recs=recs, ns=ns, n=0, lstride=32, max_n=20, count=count,
                    seed=f"counter hash 0x{seed_base + 2 + 1000 * rank:X}",
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
        return dict(name=name, recs=recs, ns=ns, n=0, lstride=32, max_n=max(large_n), count=len(ns),
                    seed=f"counter hash 0x{seed_base:X} + 4/5 + n",
                    desc=f"large single instances: n={','.join(map(str, large_n))} x ({' + '.join(kinds)})")
    raise ValueError(name)


def workload_config(wl) -> dict:
    """The `config` object of the JSON line: identical in both arms."""
    rec_bytes = 2 * wl["lstride"] + (1 if wl["ns"] is not None else 0)
    return {"workload": wl["desc"], "automata_per_gpu": wl["count"], "n": wl["n"] or f"mixed, <= {wl['max_n']}",
            "seed": wl["seed"], "record_bytes": rec_bytes, "word_stride_u64": word_stride_for(wl["max_n"]),
            "l2": L2_NOTE, "parallelism": "automata sharded by rank, no collective on the data path"}


def word_stride_for(max_n: int) -> int:
    return max(1, ((max(max_n, 2) - 1) ** 2 + 63) // 64)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class NvmlClockSampler:
    """SM clock and clock-event reasons read through NVML every `period` seconds
    on a background thread while the timed steps run (reads only: nothing about
    the GPU is set).  The timed region of the default workload lasts ~12 ms,
    shorter than nvidia-smi takes to start, so polling NVML is what places the
    samples inside it."""

    def __init__(self, gpu_index: int, period: float = 0.0005):
        import pynvml
        self.nv = pynvml
        pynvml.nvmlInit()
        self.h = pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
        self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        self.period = period
        self.samples = []
        self.done = threading.Event()
        # hand the interpreter lock over often enough for the poller to run
        # while the main thread enqueues steps (the device times are unaffected:
        # the host runs ahead of the GPU)
        self.switch = sys.getswitchinterval()
        sys.setswitchinterval(min(self.switch, period / 5))
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        nv = self.nv
        while True:
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)))
            except nv.NVMLError:
                pass
            if self.done.wait(self.period):
                return

    def stop(self):
        self.done.set()
        self.thread.join()
        sys.setswitchinterval(self.switch)
        nv = self.nv
        try:
            nv.nvmlShutdown()
        except nv.NVMLError:
            pass
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted({name for _, r in self.samples for name, b in bits.items() if r & b})
        sm = [s for s, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(self.max),
                "reasons": reasons, "samples": len(sm), "source": "NVML, polled during the timed steps"}


def clock_sampler(gpu_index: int):
    """NVML polling when the bindings load, else nvidia-smi."""
    try:
        return NvmlClockSampler(gpu_index)
    except Exception:
        return ClockSampler(gpu_index)


class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
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
# ranks
# ---------------------------------------------------------------------------

def self_launch(args, argv) -> int:
    """`--gpus N` outside torchrun: start N ranks (one process per GPU) with
    torch.distributed.run on 127.0.0.1 and pass their output through."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + list(argv)
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", "1")
    return subprocess.call(cmd, env=env)


def max_over_ranks(dist, x: float, device=None) -> float:
    """Max of a per-rank float over the process group (identity without one)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU legs (oracle restatement of the reference's CPU solver)
# ---------------------------------------------------------------------------

def cpu_pass(wl, threads: int, lengths: bool = False):
    """One pass of the CPU restatement over the workload: SlimCPU4bits13
    (uniform n <= 16, Verify mode) or SlimCPUUntweaked (otherwise)."""
    import oracle
    if wl["ns"] is None and wl["n"] <= 16:
        r = oracle.verify4(wl["recs"], n=wl["n"], lstride=wl["lstride"], write_len=lengths, threads=threads)
        kind = "SlimCPU4bits13 (nibble table, Verify mode)"
    else:
        r = oracle.solve(wl["recs"], ns=wl["ns"], n=wl["n"], lstride=wl["lstride"], words=False, threads=threads)
        kind = "SlimCPUUntweaked (lengths)"
    return r, kind


def cpu_throughput(wl, seconds: float, threads: int):
    """Passes of the CPU restatement over the workload until `seconds` of wall time."""
    t0 = time.perf_counter()
    passes = 0
    while True:
        _, kind = cpu_pass(wl, threads)
        passes += 1
        if time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return wl["count"] * passes / dt, dt, passes, kind


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle

    oracle.build()
    wl = make_workload(args.workload, args.count, 0, tuple(int(x) for x in args.large_n.split(",")),
                       tuple(args.large_kinds.split(",")), args.inputs, gen="oracle")
    threads = os.cpu_count() or 1
    for _ in range(max(args.warmup, 0)):
        cpu_pass(wl, threads)
    step_ms = []
    kind = ""
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, kind = cpu_pass(wl, threads)
        step_ms.append((time.perf_counter() - t0) * 1e3)
    ms = statistics.mean(step_ms)
    value = wl["count"] / (ms / 1e3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16", "data": "synthetic", "impl": "reference",
        "config": workload_config(wl),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} passes over the full {wl['count']:,}-automaton batch "
                                   f"({kind}, C restatement; the C# reference cannot run here); batch from "
                                   "the restatement's own System.Random"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def load_profile_json(name: str) -> dict:
    """A committed ncu / microbenchmark summary under profiles/ (or {})."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", name)))
    except (OSError, ValueError):
        return {}


def load_traffic(kernel: str):
    """DRAM bytes per launch from the committed ncu summary of this kernel, if any."""
    ent = load_profile_json("traffic.json").get(kernel)
    return ent.get("dram_bytes_per_launch") if isinstance(ent, dict) else None


class DeviceLeg:
    """Device-resident solve of one workload: records, lengths, words and the
    violation word in HBM, all work on one stream."""

    def __init__(self, eng, wl, dev, stream):
        import torch
        self.eng, self.wl, self.stream = eng, wl, stream
        self.ws = word_stride_for(wl["max_n"])
        self.d_maps = torch.from_numpy(wl["recs"]).to(dev)
        self.d_ns = torch.from_numpy(wl["ns"]).to(dev) if wl["ns"] is not None else None
        self.d_len = torch.empty(wl["count"], dtype=torch.int32, device=dev)
        self.d_words = torch.empty((wl["count"], self.ws), dtype=torch.int64, device=dev)
        self.d_fv = torch.empty(1, dtype=torch.int64, device=dev)

    def step(self):
        wl = self.wl
        self.eng.solve_device(self.d_maps, wl["lstride"], wl["count"], n=wl["n"], d_ns=self.d_ns,
                              max_n=wl["max_n"], d_len=self.d_len, d_words=self.d_words, word_stride=self.ws,
                              d_first_violation=self.d_fv, stream=self.stream)

    def timed(self, steps: int, warmup: int, flush, barrier=None, sampler_factory=None):
        """Per-step device times (ms) with L2 flushed before every step, the
        last step's statistics and the clock summary (when sampled)."""
        import torch
        for i in range(warmup):
            flush.fill_(i)
            self.step()
            self.eng.wait_device()
        sampler = sampler_factory() if sampler_factory else None
        if barrier:
            barrier()
        else:
            torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.fill_(i + 1)                 # untimed: evicts the records from L2
            evs[i][0].record(self.stream)
            self.step()
            evs[i][1].record(self.stream)
        if barrier:
            barrier()
        else:
            torch.cuda.synchronize()
        stats = self.eng.wait_device()
        clk = sampler.stop() if sampler else None
        return [a.elapsed_time(b) for a, b in evs], stats, clk


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
    props = torch.cuda.get_device_properties(dev)
    wl = make_workload(args.workload, args.count, rank, tuple(int(x) for x in args.large_n.split(",")),
                       tuple(args.large_kinds.split(",")), args.inputs)
    count, lstride = wl["count"], wl["lstride"]
    ws = word_stride_for(wl["max_n"])
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

    # ---- device-resident leg ------------------------------------------------
    # a dedicated stream: the events, the L2 flush and the library's kernels all
    # go on it (the legacy default stream would hand the library a NULL stream)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    leg = DeviceLeg(eng, wl, dev, stream)
    visible = [v for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip().isdigit()]
    gpu_index = int(visible[dev.index]) if dev.index < len(visible) else dev.index
    step_ms, stats, clk = leg.timed(args.steps, args.warmup, flush, barrier,
                                    (lambda: clock_sampler(gpu_index)) if rank == 0 else None)
    ms = statistics.mean(step_ms)
    ms_max = max_over_ranks(dist, ms, dev)
    value = count * world / (ms_max / 1e3)
    launches_per_step = int(stats.get("launches", 0))
    expanded_per_step = int(stats.get("expanded", 0))
    fv = int(leg.d_fv.item())
    lens = leg.d_len.cpu().numpy()
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
        e2e_mean = max_over_ranks(dist, statistics.mean(e2e_ms), dev)
        st = r["stats"]
        e2e = {"value": count * world / (e2e_mean / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(st["h2d_bytes"]), "d2h_bytes_per_step": int(st["d2h_bytes"]),
               "ms_per_step": e2e_mean,
               "latency_ms": {"p50": statistics.median(e2e_ms),
                              "p99": sorted(e2e_ms)[min(len(e2e_ms) - 1, int(0.99 * len(e2e_ms)))]}}
        if not np.array_equal(r["len"], lens):
            raise SystemExit("host and device paths disagree")
        # the same call with pageable (numpy) buffers: records and results pass
        # through pinned staging that host threads copy chunk by chunk
        g_len = np.empty(count, dtype=np.int32)
        g_words = np.empty((count, ws), dtype=np.uint64)
        g_ns = None if wl["ns"] is None else np.ascontiguousarray(wl["ns"])
        for i in range(min(args.warmup, 2)):
            eng.solve(wl["recs"], ns=g_ns, n=wl["n"], lstride=lstride, word_stride=ws, out=(g_len, g_words))
        pg_ms = []
        for i in range(min(args.steps, 10)):
            flush.fill_(i + 11)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            eng.solve(wl["recs"], ns=g_ns, n=wl["n"], lstride=lstride, word_stride=ws, out=(g_len, g_words))
            pg_ms.append((time.perf_counter() - t0) * 1e3)
        if not np.array_equal(g_len, lens):
            raise SystemExit("pageable and device paths disagree")
        pg_mean = max_over_ranks(dist, statistics.mean(pg_ms), dev)
        e2e["pageable"] = {"value": count * world / (pg_mean / 1e3), "unit": UNIT, "ms_per_step": pg_mean,
                           "steps": len(pg_ms), "buffers": "pageable numpy arrays (staged through pinned memory)"}

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
    threads = os.cpu_count() or 1
    if rank == 0 and world == 1:
        rate, dt, passes, kind = cpu_throughput(wl, args.cpu_seconds, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{passes} passes over the same {count:,}-automaton batch in {dt:.2f} s wall "
                         f"({kind}; C restatement, the C# reference cannot run here)"}

    line = None
    if rank == 0:
        # roofline of the dominant kernel (the step is one BFS launch plus tiny bookkeeping)
        cls = [c for c in plan.get("classes", []) if c["max_n"] >= wl["max_n"]][:1]
        kernel = cls[0]["kernel"] if cls else "k_pool"
        if cls and wl["ns"] is None and wl["n"] == 13 and cls[0].get("uniform_n13"):
            kernel = cls[0]["uniform_n13"]     # a uniform n = 13 batch runs on the per-lane kernel
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback 6.65 TB/s"
        rec_bytes = 2 * lstride + (1 if wl["ns"] is not None else 0)
        io_bytes = count * (rec_bytes + 4 + 8 * ws)
        sm_clock_mhz = (clk or {}).get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)
        onchip_cal = load_profile_json("onchip.json")
        smem_bpc = onchip_cal.get("smem_bytes_per_clk_per_sm")
        smem_src = (f"measured {smem_bpc:.1f} B/clk/SM ({onchip_cal.get('source', 'profiles/onchip.json')}) x "
                    f"{props.multi_processor_count} SMs x sampled SM clock") if smem_bpc else \
            f"nominal {NOMINAL_SMEM_BYTES_PER_CLK} B/clk/SM x {props.multi_processor_count} SMs x sampled SM clock"
        smem_peak = props.multi_processor_count * (smem_bpc or NOMINAL_SMEM_BYTES_PER_CLK) * sm_clock_mhz / 1e3
        io = {"bound": "hbm", "achieved": io_bytes / (ms / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
              "frac": io_bytes / (ms / 1e3) / 1e9 / hbm_peak, "algorithmic_bytes_per_launch": io_bytes,
              "algorithmic_bytes": "records in + lengths and words out", "peak_source": hbm_src}
        kcal = onchip_cal.get("kernels", {}).get(kernel.split("+")[0], {})
        if kernel == "k_level":
            search = expanded_per_step * LEVEL_BYTES_PER_EXPANSION
            achieved = (search + io_bytes) / (ms / 1e3) / 1e9
            roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                        "frac": achieved / hbm_peak, "traffic": load_traffic(kernel), "peak_source": hbm_src,
                        "algorithmic_bytes_per_launch": search + io_bytes,
                        "algorithmic_bytes": f"records + results + {LEVEL_BYTES_PER_EXPANSION} B per expansion "
                                             "(HBM bitmaps and queues)",
                        "expansions_per_launch": expanded_per_step}
            l2_peak = onchip_cal.get("l2_random_atomic_gops")
            atom = 2 * expanded_per_step / (ms / 1e3) / 1e9
            roofline["l2_atomics"] = {"achieved": atom, "peak": l2_peak, "unit": "G atomicOr/s",
                                      "frac": atom / l2_peak if l2_peak else None, "per_expansion": 2,
                                      "peak_source": "measured random atomicOr on an L2-resident 32 MiB bitmap "
                                                     "(profiles/onchip.json)"}
        else:
            achieved = expanded_per_step * SMEM_BYTES_PER_EXPANSION / (ms / 1e3) / 1e9
            roofline = {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                        "frac": achieved / smem_peak, "traffic": load_traffic(kernel), "peak_source": smem_src,
                        "bytes_per_expansion": SMEM_BYTES_PER_EXPANSION,
                        "expansions_per_launch": expanded_per_step,
                        "algorithmic_bytes": "28 B of shared-memory traffic per expansion (4 pop + 2 x (4 + 4) "
                                             "bitmap-word read-modify-write + 2 x 4 push)",
                        "hbm_io": io}
        if kcal:
            roofline["issue_slots_busy"] = kcal.get("issue_active")
            roofline["warps_per_sm"] = kcal.get("warps_per_sm")
            roofline["ncu_source"] = kcal.get("source")
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16", "data": "synthetic",
            "config": workload_config(wl),
            "kernel": kernel,
            "e2e": e2e,
            "roofline": roofline,
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
        if args.workload == "n12" and world == 1:
            if not args.no_serving:
                def brief(e):
                    return {"offered_per_s": e["offered_per_s"], "achieved_per_s": e["achieved_automata_per_s"],
                            "p50_ms_n_le_20": e["latency_ms_n_le_20"]["p50"],
                            "p99_ms_n_le_20": e["latency_ms_n_le_20"]["p99"],
                            "p99_ms_all": e["latency_ms"]["p99"], "client_lag_ms_p99": e["client_lag_ms_p99"],
                            "peak_hbm_admitted_bytes": e["peak_arena_bytes"] + e["peak_small_footprint_bytes"],
                            "statuses_ok": e["statuses_ok"]}
                # 100K requests at two Poisson rates and as one burst, then a 10K burst
                sweep = serve_sweep(args.serving_requests, [32000.0, 256000.0, 0.0])
                sweep += serve_sweep(10_000, [0.0])
                line["serving"] = {"requests": args.serving_requests,
                                   "sweep": [dict(brief(e), requests=e["requests"]) for e in sweep],
                                   "full_sweep": "bench.py --workload serving"}
            if not args.no_extra:
                line.update(extra_summaries(args, eng, dev, stream, flush, hbm_peak, threads))
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


def extra_summaries(args, eng, dev, stream, flush, hbm_peak: float, threads: int) -> dict:
    """The other configurations, each device-timed (L2 flushed before every
    step) with its CPU restatement beside it and its lengths compared with it."""
    import numpy as np
    import torch
    out = {}
    steps, warm = max(args.extra_steps, 1), 3

    def cpu_leg(wl):
        t0 = time.perf_counter()
        r, kind = cpu_pass(wl, threads, lengths=True)
        dt = time.perf_counter() - t0
        return r["len"], {"value": wl["count"] / dt, "unit": UNIT, "cores": threads, "kind": "port",
                          "sample": f"one pass over the {wl['count']:,} automata ({kind})"}

    # config 3: 200K automata, n uniform 6..20, 1 % Cerny
    wl = make_workload("mixed")
    leg = DeviceLeg(eng, wl, dev, stream)
    ms_l, st, _ = leg.timed(steps, warm, flush)
    ms = statistics.mean(ms_l)
    ref, cpu = cpu_leg(wl)
    out["mixed"] = {"workload": wl["desc"], "ms_per_step": ms, "automata_per_s": wl["count"] / (ms / 1e3),
                    "expansions_per_step": int(st["expanded"]), "gpu_launches_per_step": int(st["launches"]),
                    "lengths_match_cpu": bool(np.array_equal(leg.d_len.cpu().numpy(), ref)),
                    "cpu_baseline": cpu, "steps": steps}
    del leg

    # config 5: n = 24, 26, 28 x (64 random + C_n + permutation-plus-merge)
    wl = make_workload("large")
    leg = DeviceLeg(eng, wl, dev, stream)
    ms_l, st, _ = leg.timed(max(2, steps // 2), 2, flush)
    ms = statistics.mean(ms_l)
    search = int(st["expanded"]) * LEVEL_BYTES_PER_EXPANSION
    gbs = search / (ms / 1e3) / 1e9
    # the bitmaps stay in L2: every image is one random atomicOr there, against the
    # measured random-atomic throughput of an L2-resident 32 MiB bitmap
    l2_peak = load_profile_json("onchip.json").get("l2_random_atomic_gops")
    atom = 2 * int(st["expanded"]) / (ms / 1e3) / 1e9
    ref, cpu = cpu_leg(wl)
    out["large"] = {"workload": wl["desc"], "ms_per_step": ms, "automata_per_s": wl["count"] / (ms / 1e3),
                    "expansions_per_step": int(st["expanded"]),
                    "hbm_search": {"achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                                   "algorithmic_bytes": f"{LEVEL_BYTES_PER_EXPANSION} B per expansion"},
                    "l2_atomics": {"achieved": atom, "peak": l2_peak, "unit": "G atomicOr/s",
                                   "frac": atom / l2_peak if l2_peak else None,
                                   "per_expansion": 2, "peak_source": "measured (profiles/onchip.json)"},
                    "lengths_match_cpu": bool(np.array_equal(leg.d_len.cpu().numpy(), ref)),
                    "cpu_baseline": cpu, "steps": max(2, steps // 2)}
    del leg

    # the reference's published configuration: n = 13, batch 2^21 (System.Random)
    wl = make_workload("n13")
    leg = DeviceLeg(eng, wl, dev, stream)
    ms_l, st, _ = leg.timed(steps, warm, flush)
    ms = statistics.mean(ms_l)
    dev_len = leg.d_len.cpu().numpy()
    del leg
    # end to end as the reference times it: one Verify call (lengths only) on host buffers
    eng.verify(wl["recs"], n=13, lstride=13)
    v_ms = []
    for i in range(steps):
        flush.fill_(i)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rv = eng.verify(wl["recs"], n=13, lstride=13)
        v_ms.append((time.perf_counter() - t0) * 1e3)
    ref, cpu = cpu_leg(wl)
    vm = statistics.mean(v_ms)
    out["n13"] = {"workload": wl["desc"], "seed": wl["seed"], "ms_per_step": ms,
                  "automata_per_s": wl["count"] / (ms / 1e3),
                  "verify_e2e": {"value": wl["count"] / (vm / 1e3), "unit": UNIT, "ms_per_step": vm,
                                 "what": "sbfs_verify_batch on host buffers (lengths only), as Program.cs:111 "
                                         "times IComputable.Verify"},
                  "lengths_match_cpu": bool(np.array_equal(dev_len, ref) and np.array_equal(rv["len"], ref)),
                  "cpu_baseline": cpu, "published": PUBLISHED_N13, "steps": steps}
    return out


# ---------------------------------------------------------------------------
# serving: open-loop Poisson arrivals of single-automaton requests
# ---------------------------------------------------------------------------

def serve_sweep(count, rates, max_batch=0, max_levels=0, max_n=24):
    """Open-loop Poisson sweep of single-automaton requests through the serving
    loop (n log-uniform 8..max_n, 5 % Cerny family); one entry per offered rate
    (0 = all submitted at once).  A client thread submits, at every moment,
    all requests whose arrival time has passed in one sbfs_server_submit_many
    call; a request's latency is its time in the server (submission to
    result) plus how late the client submitted it after its arrival."""
    import threading

    import numpy as np

    from sbfs import problem as P
    from sbfs.server import Server

    seed = 0x5EED + 3
    ns = P.log_uniform_sizes(count, 8, max_n, seed)
    recs = P.uniform_maps(count, ns, seed + 1)
    cerny = np.arange(0, count, 20)          # 5% Cerny family
    for i in cerny:
        recs[i] = P.cerny_record(int(ns[i]))
    rng = np.random.default_rng(seed)
    sweep = []
    srv = Server(device=0, max_batch=max_batch, max_levels=max_levels, queue_capacity=max(1 << 20, 2 * count))

    def collect(want, t_limit):
        got = []
        have = 0
        while have < want:
            a = srv.poll_array(timeout_ms=20)
            if a.size:
                got.append(a)
                have += a.size
            elif time.perf_counter() > t_limit:
                raise SystemExit("serving run did not finish")
        return np.concatenate(got) if got else np.zeros(0)

    # warm-up: the whole request set once, so every kernel the sweep uses has been
    # loaded and launched before anything is timed
    srv.submit_many(recs, ns)
    collect(count, time.perf_counter() + 600)
    for rate in rates:
        srv.reset_peak()
        gaps = rng.exponential(1.0 / rate, count) if rate > 0 else np.zeros(count)
        arrive = np.cumsum(gaps)
        ids = np.zeros(count, dtype=np.uint64)
        lag = np.zeros(count)
        retries = [0]

        def submitter():
            t0 = time.perf_counter()
            i = 0
            while i < count:
                now = time.perf_counter() - t0
                j = int(np.searchsorted(arrive, now, side="right"))
                if j <= i:
                    wait = arrive[i] - now
                    if wait > 2e-4:
                        time.sleep(wait * 0.5)
                    continue
                try:
                    ids[i:j] = srv.submit_many(recs[i:j], ns[i:j])
                except Exception:
                    retries[0] += 1
                    time.sleep(1e-4)
                    continue
                lag[i:j] = (time.perf_counter() - t0) - arrive[i:j]
                i = j

        th = threading.Thread(target=submitter)
        t_start = time.perf_counter()
        th.start()
        res = collect(count, t_start + 600)
        th.join()
        wall = time.perf_counter() - t_start
        st = srv.stats()
        order = np.argsort(res["id"])
        res = res[order]
        pos = np.searchsorted(res["id"], ids)
        res = res[pos]                      # in submission order
        lat = (res["done_ms"] - res["submit_ms"]) + lag * 1e3
        n_of = res["n"]
        small = n_of <= 20
        tiny = n_of <= 16
        mid = small & ~tiny
        span_ms = float(res["done_ms"].max() - res["submit_ms"].min())
        entry = {
            "offered_per_s": rate if rate > 0 else "all at once",
            "requests": count,
            "achieved_automata_per_s": count / (span_ms / 1e3),
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "latency_ms_n_le_20": {"p50": float(np.percentile(lat[small], 50)),
                                   "p99": float(np.percentile(lat[small], 99))},
            "latency_ms_n_le_16": {"p50": float(np.percentile(lat[tiny], 50)),
                                   "p99": float(np.percentile(lat[tiny], 99))},
            "latency_ms_n_17_20": {"p50": float(np.percentile(lat[mid], 50)),
                                   "p99": float(np.percentile(lat[mid], 99))},
            "client_lag_ms_p99": float(np.percentile(lag, 99) * 1e3),
            "peak_arena_bytes": int(st["arena_peak"]), "peak_small_footprint_bytes": int(st["small_peak"]),
            "statuses_ok": bool((res["status"] == 0).all()),
            "submit_retries": retries[0], "wall_s": wall,
        }
        sweep.append(entry)
        print(json.dumps({"serving_rate": entry}), file=sys.stderr, flush=True)
    srv.stop()
    return sweep


def run_serving(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    count = args.count or 100_000
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


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    args = parse_args(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return self_launch(args, argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)
    return run_sbfs(args)


if __name__ == "__main__":
    sys.exit(main())

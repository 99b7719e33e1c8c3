"""bench.py's rank plumbing on CPU: `--gpus N` outside torchrun starts N ranks
itself and rank 0 prints exactly one JSON line with n_gpus = N; the max over
ranks that every multi-GPU time goes through, on two gloo ranks; and the
reference arm's config object is the GPU arm's (same keys and values)."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_gpus_two_self_launches_two_ranks():
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "n8", "--count", "3000", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["n_gpus"] == 2 and line["impl"] == "reference"
    assert line["config"]["automata_per_gpu"] == 3000
    # the launcher started two ranks (torchrun reports both workers' exits)
    assert "WORLD_SIZE" not in env


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out_dir):
    import datetime
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    got = bench.max_over_ranks(dist, 1.5 + rank * 2.25, None)
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(repr(got))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_two_gloo_ranks(tmp_path):
    mp.start_processes(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert [float(open(tmp_path / f"r{r}.txt").read()) for r in range(2)] == [3.75, 3.75]


def test_both_arms_share_one_config():
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    for name in ("n8", "n12", "mixed"):
        a = bench.make_workload(name, count=500, gen="oracle")    # the reference arm's batch
        b = bench.make_workload(name, count=500, gen="sbfs")      # the GPU arm's batch
        np.testing.assert_array_equal(a["recs"], b["recs"])
        assert bench.workload_config(a) == bench.workload_config(b)
        assert set(bench.workload_config(a)) == {"workload", "automata_per_gpu", "n", "seed", "record_bytes",
                                                 "word_stride_u64", "l2", "parallelism"}

"""Shared-memory throughput per SM clock on this GPU: the measured denominator
of the on-chip roofline that bench.py reports for the BFS kernels (28 B of
shared-memory traffic per expansion).  tests/cuda/smem_peak.cu is built with
nvcc for sm_100a and run with one 1024-thread CTA per SM: lane-interleaved
32-bit loads (each warp access on 32 banks) and 32-bit shared atomicOr.  The
figures are printed (and written to $SBFS_SMEM_PEAK_OUT when set) so they can
be recorded beside the ncu summaries; the test bounds them by the hardware's
32 banks x 4 B per clock."""
import ctypes
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_shared_memory_bytes_per_clock(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    torch.cuda.synchronize()
    so = str(tmp_path / "smem_peak.so")
    subprocess.check_call(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared",
                           "-Xcompiler", "-fPIC", "-o", so, os.path.join(HERE, "cuda", "smem_peak.cu")])
    lib = ctypes.CDLL(so)
    lib.smem_bytes_per_clk.argtypes = [ctypes.c_int, ctypes.c_int]
    lib.smem_bytes_per_clk.restype = ctypes.c_double
    loads = lib.smem_bytes_per_clk(0, 4096)
    atomics = lib.smem_bytes_per_clk(1, 1024)
    out = {"smem_load_bytes_per_clk_per_sm": loads, "smem_atomic_or_bytes_per_clk_per_sm": atomics,
           "device": torch.cuda.get_device_name(0), "sms": torch.cuda.get_device_properties(0).multi_processor_count}
    print(json.dumps(out))
    if os.environ.get("SBFS_SMEM_PEAK_OUT"):
        with open(os.environ["SBFS_SMEM_PEAK_OUT"], "w") as f:
            json.dump(out, f)
    assert 32.0 <= loads <= 128.5
    assert 4.0 <= atomics <= 128.5

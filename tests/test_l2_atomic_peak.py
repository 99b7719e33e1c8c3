"""Random 32-bit atomicOr throughput on an L2-resident 32 MiB bitmap: the
measured roof of the level engine's wide levels (n = 21..28), whose every image
costs one such test-and-set on the automaton's bitmap.  tests/cuda/
l2_atomic_peak.cu is built with nvcc for sm_100a and run with four independent
atomics in flight per thread; the figure is printed (and written to
$SBFS_L2_PEAK_OUT when set) so it can be recorded beside the ncu summaries."""
import ctypes
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def test_random_l2_atomics_per_second(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    torch.cuda.synchronize()
    so = str(tmp_path / "l2_atomic_peak.so")
    subprocess.check_call(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-shared",
                           "-Xcompiler", "-fPIC", "-o", so, os.path.join(HERE, "cuda", "l2_atomic_peak.cu")])
    lib = ctypes.CDLL(so)
    lib.l2_random_atomic_gops.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.l2_random_atomic_gops.restype = ctypes.c_double
    out = {f"ctas_per_sm_{c}": lib.l2_random_atomic_gops(23, c, 256) for c in (2, 4)}   # 2^23 words = 32 MiB
    out["g_atomics_per_s"] = max(out.values())
    out["device"] = torch.cuda.get_device_name(0)
    print(json.dumps(out))
    if os.environ.get("SBFS_L2_PEAK_OUT"):
        with open(os.environ["SBFS_L2_PEAK_OUT"], "w") as f:
            json.dump(out, f)
    assert out["g_atomics_per_s"] > 1.0

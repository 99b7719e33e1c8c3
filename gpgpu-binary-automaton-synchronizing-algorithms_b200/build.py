"""Builds libsbfs.so (the CUDA engine behind include/sbfs.h) in-tree for sm_100a.

    python build.py            # incremental
    python build.py --force    # rebuild everything

Objects go to _build/ next to this file; the library to sbfs/_lib/libsbfs.so.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "sbfs", "_lib")
LIB = os.path.join(LIBDIR, "libsbfs.so")
CHECKED_LIB = os.path.join(LIBDIR, "libsbfs_checked.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                     "-I", INCLUDE, "-I", CSRC, "--expt-relaxed-constexpr"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith((".h", ".hpp"))]
    return hs


def _compile(src: str, obj: str, extra):
    cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False, extra=(), checked: bool = False) -> str:
    """Compiles the library; checked=True builds libsbfs_checked.so instead, with
    -DSBFS_CHECKED (data-derived indices checked on the device, failures
    reported as an error status; see csrc/common.cuh)."""
    build_dir = os.path.join(BUILD, "checked") if checked else BUILD
    lib = CHECKED_LIB if checked else LIB
    extra = list(extra) + (["-DSBFS_CHECKED"] if checked else [])
    os.makedirs(build_dir, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    newest_header = max((os.path.getmtime(h) for h in _headers()), default=0)
    jobs = []
    objs = []
    for f in srcs:
        src = os.path.join(CSRC, f)
        obj = os.path.join(build_dir, f[:-3] + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src),
                                                                                 newest_header)
        if stale:
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            futs = {ex.submit(_compile, s, o, extra): s for s, o in jobs}
            for fu in cf.as_completed(futs):
                msg = fu.result()
                if verbose and msg:
                    print(msg, file=sys.stderr)
    if jobs or not os.path.exists(lib) or force:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    force = "--force" in sys.argv
    verbose = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(force=force, verbose=verbose or bool(extra), extra=extra, checked="--checked" in sys.argv))

"""sbfs -- exact shortest synchronizing words of binary automata on B200.

Python face of libsbfs.so (include/sbfs.h).  The compute path is the CUDA
library only; importing this package never falls back to a CPU solver.
"""
from .problem import (Problem, generate_worst_case, uniform_maps, uniform_sizes, log_uniform_sizes,
                      cerny_record, perm_merge_record, records_from_problems, problems_from_records,
                      repack, RECORD_LSTRIDE, MAX_N)
from .solver import (Engine, SlimGPUNative, ComputationResult, word_stride_for, word_bits_to_bools,
                     verify_and_report, read_cerny_failed)
from . import dotnet_random
from ._native import load, NativeUnavailable, SbfsError, LIB_PATH, EXPORTS

__all__ = [
    "Problem", "generate_worst_case", "uniform_maps", "uniform_sizes", "log_uniform_sizes",
    "cerny_record", "perm_merge_record", "records_from_problems", "problems_from_records", "repack",
    "RECORD_LSTRIDE", "MAX_N", "Engine", "SlimGPUNative", "ComputationResult", "word_stride_for",
    "word_bits_to_bools", "verify_and_report", "read_cerny_failed", "dotnet_random", "load",
    "NativeUnavailable", "SbfsError", "LIB_PATH", "EXPORTS",
]

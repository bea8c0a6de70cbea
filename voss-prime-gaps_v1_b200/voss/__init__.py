"""voss — B200-native wheel-30 sieve, gap statistics and Miller-Rabin verification.

A drop-in for the sieve/extract/gap stages of VOSS (src/voss_v7_live.cu) and for its
verifier (src/verify_cpp.cpp): the compute runs in libvoss.so (hand-written sm_100a CUDA
behind a C ABI, include/voss.h); this package is its ctypes face.
"""
from ._native import (FLAG_REF_COMPAT, IHIST, MAX_GAP, MODQ_MAX_GAP, Q_LIST, VossError, lib_path,  # noqa: F401
                      load)
from .api import (INTERVAL_DTYPE, LARGE_DTYPE, Context, RangeResult, device_count, merge_stats,  # noqa: F401
                  range_result, run_checkpointed_fn, to_struct, version, write_artifacts, write_gap_sequence)

__all__ = [
    "Context", "RangeResult", "VossError", "merge_stats", "write_artifacts", "device_count", "version",
    "FLAG_REF_COMPAT", "INTERVAL_DTYPE", "LARGE_DTYPE", "MAX_GAP", "MODQ_MAX_GAP", "Q_LIST", "IHIST",
]

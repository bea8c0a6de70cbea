"""ctypes binding of libvoss.so (the C ABI declared in include/voss.h).

The library is loaded from voss/_lib/libvoss.so next to this file, or from the path in the
VOSS_LIB environment variable.  There is no fallback: if the library cannot be loaded every
call raises VossError, so a missing build can never silently run something else.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_uint8, c_uint32, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(HERE, "_lib", "libvoss.so")

# ---- constants mirrored from include/voss.h ------------------------------------------
VOSS_OK = 0
ERRORS = {
    -1: "VOSS_ERR_ARG", -2: "VOSS_ERR_CUDA", -3: "VOSS_ERR_NOMEM", -4: "VOSS_ERR_RANGE",
    -5: "VOSS_ERR_DEVICE", -6: "VOSS_ERR_TIMEOUT", -7: "VOSS_ERR_STOPPED", -8: "VOSS_ERR_IO",
    -9: "VOSS_ERR_STATE", -10: "VOSS_ERR_NODEV",
}
MAX_GAP = 100000
MODQ_MAX_GAP = 100
MODQ_ROWS = 10
NUM_Q = 10
MODQ_SLOTS = 99
Q_LIST = (3, 4, 5, 6, 7, 8, 11, 12, 13, 30)
IHIST = 1024
FLAG_REF_COMPAT = 1


class VossError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class LargeGap(ctypes.Structure):
    _fields_ = [("position", c_uint64), ("gap", c_int32), ("merit", c_float)]


class RangeStats(ctypes.Structure):
    _fields_ = [
        ("lo", c_uint64), ("hi", c_uint64), ("flags", c_uint32), ("reserved0", c_uint32),
        ("seg_num", c_uint64), ("prime_count", c_uint64), ("first_prime", c_uint64),
        ("last_prime", c_uint64), ("max_gap", c_uint64), ("max_gap_lo", c_uint64),
        ("mod4", c_uint64 * 2), ("modq", c_uint64 * MODQ_SLOTS),
        ("modq_gap", (c_uint64 * MODQ_MAX_GAP) * MODQ_ROWS), ("large_total", c_uint64),
        ("gap_hist", c_uint64 * MAX_GAP),
    ]


class IntervalStats(ctypes.Structure):
    _fields_ = [
        ("lo", c_uint64), ("hi", c_uint64), ("prime_count", c_uint64), ("first_prime", c_uint64),
        ("last_prime", c_uint64), ("max_gap", c_uint64), ("max_gap_lo", c_uint64),
        ("gap_overflow", c_uint64), ("gap_hist", c_uint64 * IHIST),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [
        ("block_threads", c_uint32), ("chunk_words", c_uint32), ("ctas_per_sm", c_uint32),
        ("coop_div", c_uint32), ("mult_factor", c_uint32), ("medium_mode", c_uint32),
        ("walk_sixteenths", c_uint32), ("mr_route", c_uint32),
    ]


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("slots", c_uint32), ("max_batch_requests", c_uint32), ("max_batch_tiles", c_uint32),
        ("fail_every_n_batches", c_uint32), ("max_batch_candidates", c_uint64), ("max_batch_bitmap_bytes", c_uint64),
        ("reserved", c_uint64 * 1),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("batches", c_uint64), ("completed", c_uint64), ("failed", c_uint64), ("pending", c_uint64),
        ("kernel_launches", c_uint64), ("max_inflight_batches", c_uint32), ("reserved0", c_uint32),
        ("mean_batch_requests", c_double),
    ]


SEGMENT_FN = ctypes.CFUNCTYPE(c_int, c_void_p, c_uint64, c_uint64, POINTER(RangeStats), POINTER(LargeGap),
                              c_uint64, POINTER(c_uint64))


# name -> (restype, argtypes); every entry point declared in include/voss.h
SIGNATURES = {
    "voss_version": (c_char_p, []),
    "voss_last_error": (c_char_p, []),
    "voss_device_count": (c_int, [POINTER(c_int)]),
    "voss_ctx_create": (c_int, [c_int, c_uint64, POINTER(c_void_p)]),
    "voss_ctx_destroy": (None, [c_void_p]),
    "voss_ctx_info": (c_int, [c_void_p, POINTER(c_uint64), POINTER(c_uint64), POINTER(c_int)]),
    "voss_ctx_set_tuning": (c_int, [c_void_p, POINTER(Tuning)]),
    "voss_ctx_get_tuning": (c_int, [c_void_p, POINTER(Tuning)]),
    "voss_sieve_range": (c_int, [c_void_p, c_uint64, c_uint64, c_uint32, c_uint64, POINTER(RangeStats),
                                 POINTER(LargeGap), c_uint64, POINTER(c_uint64)]),
    "voss_sieve_range_device": (c_int, [c_void_p, c_uint64, c_uint64, c_uint32, c_uint64, c_void_p]),
    "voss_fetch_range": (c_int, [c_void_p, POINTER(RangeStats), POINTER(LargeGap), c_uint64, POINTER(c_uint64)]),
    "voss_gaps_at_least": (c_int, [c_void_p, c_uint64, c_uint64, c_uint32, POINTER(LargeGap), c_uint64,
                                   POINTER(c_uint64)]),
    "voss_primes_range": (c_int, [c_void_p, c_uint64, c_uint64, POINTER(c_uint64), c_uint64, POINTER(c_uint64)]),
    "voss_sieve_intervals": (c_int, [c_void_p, POINTER(c_uint64), POINTER(c_uint64), c_uint32,
                                     POINTER(IntervalStats)]),
    "voss_mr_verify": (c_int, [c_void_p, POINTER(c_uint64), c_uint64, POINTER(c_uint8)]),
    "voss_mr_verify_device": (c_int, [c_void_p, c_void_p, c_uint64, c_void_p, c_void_p]),
    "voss_mr_verify_noalloc": (c_int, [c_void_p, c_uint64, c_void_p, c_void_p]),
    "voss_prove_gaps": (c_int, [c_void_p, POINTER(c_uint64), POINTER(c_int32), c_uint64, POINTER(c_uint8)]),
    "voss_sha256_batch": (c_int, [c_void_p, POINTER(c_uint8), POINTER(c_uint64), c_uint64, POINTER(c_uint8)]),
    "voss_write_artifacts": (c_int, [POINTER(RangeStats), POINTER(LargeGap), c_uint64, c_char_p]),
    "voss_stats_merge": (c_int, [POINTER(RangeStats), c_uint32, POINTER(RangeStats), POINTER(LargeGap),
                                 c_uint64, c_uint64, POINTER(c_uint64)]),
    "voss_gap_sequence": (c_int, [c_void_p, c_uint64, c_uint64, c_uint64, POINTER(c_int32), POINTER(c_uint64),
                                  POINTER(c_uint64)]),
    "voss_write_gap_sequence": (c_int, [POINTER(c_int32), POINTER(c_uint64), c_uint64, c_char_p]),
    "voss_run_checkpointed": (c_int, [c_void_p, c_uint64, c_uint64, c_uint32, c_uint32, c_char_p, POINTER(RangeStats),
                                      POINTER(LargeGap), c_uint64, POINTER(c_uint64), POINTER(c_uint64)]),
    "voss_run_checkpointed_fn": (c_int, [SEGMENT_FN, c_void_p, c_uint64, c_uint64, c_uint32, c_uint32, c_char_p,
                                         POINTER(RangeStats), POINTER(LargeGap), c_uint64, POINTER(c_uint64),
                                         POINTER(c_uint64)]),
    "voss_server_create": (c_int, [c_void_p, POINTER(ServerConfig), POINTER(c_void_p)]),
    "voss_server_destroy": (None, [c_void_p]),
    "voss_server_submit_interval": (c_int, [c_void_p, c_uint64, c_uint64, POINTER(c_uint64)]),
    "voss_server_submit_mr": (c_int, [c_void_p, POINTER(c_uint64), c_uint64, POINTER(c_uint64)]),
    "voss_server_wait": (c_int, [c_void_p, c_uint64, c_uint32]),
    "voss_server_result_interval": (c_int, [c_void_p, c_uint64, POINTER(IntervalStats)]),
    "voss_server_result_mr": (c_int, [c_void_p, c_uint64, POINTER(c_uint8), c_uint64]),
    "voss_server_request_times": (c_int, [c_void_p, c_uint64, POINTER(c_double), POINTER(c_double), POINTER(c_double)]),
    "voss_server_release": (c_int, [c_void_p, c_uint64]),
    "voss_server_get_stats": (c_int, [c_void_p, POINTER(ServerStats)]),
    "voss_probe_smem_rmw": (c_int, [c_void_p, POINTER(c_double)]),
    "voss_last_kernel_ms": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double)]),
    "voss_last_phase_ms": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double), POINTER(c_double),
                                   POINTER(c_uint32)]),
    "voss_probe_mulmod": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double)]),
}

_lib = None
_lib_path = None


def lib_path() -> str:
    return os.environ.get("VOSS_LIB") or DEFAULT_LIB


def load(path: str | None = None) -> ctypes.CDLL:
    """Load libvoss.so once and bind every signature; raises VossError if it is missing."""
    global _lib, _lib_path
    p = path or lib_path()
    if _lib is not None and _lib_path == p:
        return _lib
    if not os.path.exists(p):
        raise VossError(-2, f"libvoss.so not built: {p} (run __graft_entry__.build() or make)")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib, _lib_path = lib, p
    return lib


def check(rc: int) -> None:
    if rc != VOSS_OK:
        msg = load().voss_last_error()
        raise VossError(rc, msg.decode() if msg else "")

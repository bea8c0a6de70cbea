"""ctypes access to the CPU oracle (oracle/liboracle.so) and to the reference verifier
compiled unmodified (oracle/_ref/libref_verify.so).  Test infrastructure: used only as the
checker, never by the product package."""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, byref, c_int, c_int32, c_uint8, c_uint32, c_uint64

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_VERIFY_SO = os.path.join(ROOT, "oracle", "_ref", "libref_verify.so")
REF_BIN_DIR = os.path.join(ROOT, "oracle", "_ref")

import sys  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "voss-prime-gaps_v1_b200"))
from voss import _native as N  # noqa: E402
from voss.api import LARGE_DTYPE, INTERVAL_DTYPE, range_result  # noqa: E402

_o = None
_r = None


def oracle():
    global _o
    if _o is None:
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_is_prime_u64.restype = c_int
        L.oracle_is_prime_u64.argtypes = [c_uint64]
        L.oracle_mr_batch.argtypes = [POINTER(c_uint64), c_uint64, POINTER(c_uint8), c_int]
        L.oracle_prove_gaps.argtypes = [POINTER(c_uint64), POINTER(c_int32), c_uint64, POINTER(c_uint8), c_int]
        L.oracle_sieve_range.restype = c_int
        L.oracle_sieve_range.argtypes = [c_uint64, c_uint64, c_uint32, c_uint64, c_int, POINTER(N.RangeStats),
                                         POINTER(N.LargeGap), c_uint64, POINTER(c_uint64)]
        L.oracle_sieve_intervals.restype = c_int
        L.oracle_sieve_intervals.argtypes = [POINTER(c_uint64), POINTER(c_uint64), c_uint32, c_int,
                                             POINTER(N.IntervalStats)]
        L.oracle_primes_range.restype = c_int
        L.oracle_primes_range.argtypes = [c_uint64, c_uint64, POINTER(c_uint64), c_uint64, POINTER(c_uint64)]
        L.oracle_sieve_work.restype = c_uint64
        L.oracle_sieve_work.argtypes = [c_uint64]
        L.oracle_max_threads.restype = c_int
        _o = L
    return _o


def ref_verify():
    global _r
    if _r is None:
        L = ctypes.CDLL(REF_VERIFY_SO)
        L.ref_is_prime_u64.restype = c_int
        L.ref_is_prime_u64.argtypes = [c_uint64]
        L.ref_mr_batch.argtypes = [POINTER(c_uint64), c_uint64, POINTER(c_uint8), c_int]
        L.ref_prove_gaps.argtypes = [POINTER(c_uint64), POINTER(c_int32), c_uint64, POINTER(c_uint8), c_int]
        L.ref_max_threads.restype = c_int
        _r = L
    return _r


def _p64(a):
    return a.ctypes.data_as(POINTER(c_uint64))


def _p8(a):
    return a.ctypes.data_as(POINTER(c_uint8))


def _p32(a):
    return a.ctypes.data_as(POINTER(c_int32))


def sieve_range(lo, hi, compat=False, seg_num=30_000_000_000, threads=0, large_cap=1 << 22):
    st = N.RangeStats()
    large = np.zeros(large_cap, dtype=LARGE_DTYPE)
    w = c_uint64()
    rc = oracle().oracle_sieve_range(lo, hi, N.FLAG_REF_COMPAT if compat else 0, seg_num if compat else 0,
                                     threads, byref(st), large.ctypes.data_as(POINTER(N.LargeGap)), large_cap,
                                     byref(w))
    assert rc == 0
    return range_result(st, large[: w.value].copy())


def sieve_intervals(lo, hi, threads=0):
    lo = np.ascontiguousarray(lo, dtype=np.uint64)
    hi = np.ascontiguousarray(hi, dtype=np.uint64)
    out = np.zeros(lo.size, dtype=INTERVAL_DTYPE)
    rc = oracle().oracle_sieve_intervals(_p64(lo), _p64(hi), lo.size, threads,
                                         out.ctypes.data_as(POINTER(N.IntervalStats)))
    assert rc == 0
    return out


def primes_range(lo, hi):
    cnt = c_uint64()
    oracle().oracle_primes_range(lo, hi, None, 0, byref(cnt))
    out = np.zeros(max(cnt.value, 1), dtype=np.uint64)
    oracle().oracle_primes_range(lo, hi, _p64(out), cnt.value, byref(cnt))
    return out[: cnt.value]


def mr_batch(n, threads=0):
    n = np.ascontiguousarray(n, dtype=np.uint64)
    out = np.zeros(n.size, dtype=np.uint8)
    oracle().oracle_mr_batch(_p64(n), n.size, _p8(out), threads)
    return out


def prove_gaps(p_after, gap, threads=0):
    p = np.ascontiguousarray(p_after, dtype=np.uint64)
    g = np.ascontiguousarray(gap, dtype=np.int32)
    out = np.zeros(p.size, dtype=np.uint8)
    oracle().oracle_prove_gaps(_p64(p), _p32(g), p.size, _p8(out), threads)
    return out


def ref_mr_batch(n, threads=0):
    n = np.ascontiguousarray(n, dtype=np.uint64)
    out = np.zeros(n.size, dtype=np.uint8)
    ref_verify().ref_mr_batch(_p64(n), n.size, _p8(out), threads)
    return out


def ref_prove_gaps(p_after, gap, threads=0):
    p = np.ascontiguousarray(p_after, dtype=np.uint64)
    g = np.ascontiguousarray(gap, dtype=np.int32)
    out = np.zeros(p.size, dtype=np.uint8)
    ref_verify().ref_prove_gaps(_p64(p), _p32(g), p.size, _p8(out), threads)
    return out


def sieve_work(n):
    return oracle().oracle_sieve_work(n)

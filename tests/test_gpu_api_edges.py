"""Argument checks and degenerate inputs of the C ABI on the GPU: every invalid call returns its
error code (never a crash or a silent result), and empty or tiny ranges give exact answers."""
import numpy as np
import pytest

import voss

pytestmark = pytest.mark.gpu

ARG, RANGE, STATE = -1, -4, -9
SEG = 30_000_000_000


def _code(fn, *a, **k):
    with pytest.raises(voss.VossError) as e:
        fn(*a, **k)
    return e.value.code


def test_invalid_arguments_return_codes():
    with voss.Context(10**9) as ctx:
        assert _code(ctx.fetch_range) == STATE                       # nothing sieved yet
        assert _code(ctx.sieve_range, 100, 50) == ARG                 # hi < lo
        assert _code(ctx.sieve_range, 1, 10**9 + 1) == RANGE          # beyond the context
        assert _code(ctx.sieve_range, 1, 10**6, compat=True, seg_num=31) == ARG   # not a multiple of 30
        assert _code(ctx.sieve_range, 1, 10**6, compat=True, seg_num=30 * 1000) == ARG  # below a tile
        assert _code(ctx.sieve_intervals, np.array([10], np.uint64), np.array([5], np.uint64)) == ARG
        assert _code(ctx.sieve_intervals, np.array([10], np.uint64), np.array([10**9 + 1], np.uint64)) == RANGE
        assert _code(ctx.set_tuning, block_threads=600) == ARG
        assert _code(ctx.set_tuning, chunk_words=48) == ARG
        assert _code(ctx.set_tuning, mult_factor=100) == ARG
        t = ctx.set_tuning()                                          # defaults still in force
        assert t["block_threads"] == 1024 and t["chunk_words"] == 49


def test_empty_and_tiny_ranges():
    with voss.Context(10**9) as ctx:
        for lo, hi, pi in [(0, 0, 0), (5, 5, 0), (0, 2, 0), (1, 2, 0), (2, 3, 1), (1, 8, 4), (0, 32, 11),
                           (7, 8, 1), (8, 11, 0), (89, 97, 1), (1, 121, 30)]:
            r = ctx.sieve_range(lo, hi)
            assert r.prime_count == pi, (lo, hi)
        iv = ctx.sieve_intervals(np.array([0, 5, 2, 1000], np.uint64), np.array([0, 5, 3, 1000], np.uint64))
        assert iv["prime_count"].tolist() == [0, 0, 1, 0]
        assert ctx.sieve_intervals(np.zeros(0, np.uint64), np.zeros(0, np.uint64)).size == 0
        assert ctx.mr_verify(np.zeros(0, np.uint64)).size == 0
        assert ctx.prove_gaps(np.zeros(0, np.uint64), np.zeros(0, np.int32)).size == 0
        assert ctx.primes_range(10, 10).size == 0
        assert ctx.primes_range(1, 30).tolist() == [2, 3, 5, 7, 11, 13, 17, 19, 23, 29]


def test_phase_times_and_kernel_counts():
    """voss_last_phase_ms splits voss_last_kernel_ms into its phases and counts the kernels."""
    with voss.Context(10**16 + 10**8) as ctx:
        ctx.sieve_range(1, 10**9 + 1)
        pre, tile, tail, k = ctx.last_phase_ms()
        sieve, total = ctx.last_kernel_ms()
        assert k == 3                                   # tile kernel, stitch, reduce (no pre-pass)
        assert min(pre, tile, tail) >= 0 and tile > 0
        assert abs(pre + tile - sieve) < 0.05 and abs(pre + tile + tail - total) < 0.05
        lo = np.array([10**15, 10**12, 10**16], dtype=np.uint64)
        hi = lo + np.array([10**7, 10**6, 10**8], dtype=np.uint64)
        ctx.sieve_intervals(lo, hi)
        pre, tile, tail, k = ctx.last_phase_ms()
        assert k >= 5                                   # >= 1 pre-pass window + tile, stitch, reduce, finalize
        assert pre > 0 and tile > 0 and tail > 0


def test_mulmod_probe_rates():
    with voss.Context(10**9) as ctx:
        full, small = ctx.probe_mulmod()
        assert 1e10 < full < 1e14 and 1e10 < small < 1e14
        assert small >= 0.9 * full                      # the n < 2^63 product skips the carry checks

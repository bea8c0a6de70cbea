"""GPU parity of the sieve-and-gap kernels (libvoss.so) against the CPU oracle and the
reference's golden vectors.  Integer work: every comparison is exact."""
import json
import os

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
SEG = 30_000_000_000


def large_key(arr):
    return sorted((int(p), int(g)) for p, g in zip(arr["position"], arr["gap"]))


def assert_range_equal(g, o, check_large=True):
    for k in ("lo", "hi", "flags", "seg_num", "prime_count", "first_prime", "last_prime", "max_gap",
              "max_gap_lo", "large_total"):
        assert getattr(g, k) == getattr(o, k), (k, getattr(g, k), getattr(o, k))
    np.testing.assert_array_equal(g.mod4, o.mod4)
    np.testing.assert_array_equal(g.modq, o.modq)
    np.testing.assert_array_equal(g.modq_gap, o.modq_gap)
    np.testing.assert_array_equal(g.gap_hist, o.gap_hist)
    if check_large:
        assert large_key(g.large) == large_key(o.large)
        # merits: device log() vs host log() may differ in the last double ulp; as floats they agree
        gm = {(int(p), int(x)): float(m) for p, x, m in zip(g.large["position"], g.large["gap"], g.large["merit"])}
        om = {(int(p), int(x)): float(m) for p, x, m in zip(o.large["position"], o.large["gap"], o.large["merit"])}
        for key, m in om.items():
            assert abs(gm[key] - m) <= 4e-6 * max(1.0, abs(m)), (key, gm[key], m)


@pytest.mark.parametrize("lo,hi", [
    (0, 0), (0, 1), (0, 2), (0, 3), (2, 3), (3, 8), (1, 8), (5, 6), (7, 8), (1, 100), (1, 1000), (1, 1001),
    (1, 10**6 + 1), (2, 10**7), (999_999_000, 1_000_001_000), (10**9, 10**9 + 10**7 + 7),
    (123_456_789, 987_654_321), (10**12 - 10**8, 10**12 + 1),
])
def test_range_full_matches_oracle(gpu_ctx, lo, hi):
    g = gpu_ctx.sieve_range(lo, hi)
    o = O.sieve_range(lo, hi)
    assert_range_equal(g, o)


@pytest.mark.parametrize("n", [7, 8, 30, 97, 1000, 10**6, 10**8, 10**9])
def test_compat_matches_oracle(gpu_ctx, n):
    g = gpu_ctx.sieve_range(1, n + 1, compat=True, seg_num=SEG)
    o = O.sieve_range(1, n + 1, compat=True, seg_num=SEG)
    assert_range_equal(g, o)


def test_compat_segment_boundary_rule(gpu_ctx):
    # a short segment length puts reference-segment seams inside and between tiles
    t = gpu_ctx.tuning()
    seg = 30 * 4 * t["block_threads"] * t["chunk_words"] * 3 + 30 * 7  # not a tile multiple
    for n in (10**8, 3 * 10**8 + 11):
        g = gpu_ctx.sieve_range(1, n + 1, compat=True, seg_num=seg)
        o = O.sieve_range(1, n + 1, compat=True, seg_num=seg)
        assert_range_equal(g, o)


def test_random_ranges_match_oracle(gpu_ctx):
    rng = np.random.default_rng(20261203)
    for _ in range(12):
        e = rng.uniform(2, 12.5)
        lo = int(10**e)
        ln = int(10 ** rng.uniform(0, 6.5))
        g = gpu_ctx.sieve_range(lo, lo + ln)
        o = O.sieve_range(lo, lo + ln)
        assert_range_equal(g, o)


def test_golden_pi_and_chebyshev(gpu_ctx):
    for n in (9, 10, 11):
        g = gpu_ctx.sieve_range(1, 10**n + 1, compat=True, seg_num=SEG)
        assert g.prime_count == GOLD["pi_10n"][str(n)]
        p41, p43 = GOLD["chebyshev"][str(10**n)]
        assert (int(g.mod4[0]), int(g.mod4[1])) == (p41, p43)
        # the reference's three self-checks (src/voss_v7_live.cu:693-705)
        gh = g.gap_hist
        assert int(gh.sum()) == g.prime_count - 1
        assert int((np.arange(gh.size, dtype=np.uint64) * gh).sum()) == g.last_prime - 2
        assert int(g.mod4.sum()) + 1 == g.prime_count


@pytest.mark.parametrize("n", [10**11, 10**12])
def test_golden_gap_histogram(gpu_ctx, n):
    g = gpu_ctx.sieve_range(1, n + 1, compat=True, seg_num=SEG)
    gold = GOLD["gap_hist"][str(n)]
    got = {str(i): int(c) for i, c in enumerate(g.gap_hist) if c}
    assert got == gold
    assert g.prime_count == GOLD["pi_10n"][str(len(str(n)) - 1)]
    assert [int(g.mod4[0]), int(g.mod4[1])] == GOLD["chebyshev"][str(n)]


def test_intervals_match_oracle_and_single_launch(gpu_ctx):
    rng = np.random.default_rng(7)
    k = 64
    lo = (10 ** rng.uniform(1, 12.5, k)).astype(np.uint64)
    ln = (10 ** rng.uniform(0, 6, k)).astype(np.uint64)
    lo[:4] = [0, 1, 2, 5]
    ln[:4] = [0, 30, 1, 1000]
    hi = lo + ln
    g = gpu_ctx.sieve_intervals(lo, hi)
    o = O.sieve_intervals(lo, hi)
    for f in ("lo", "hi", "prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "gap_overflow"):
        np.testing.assert_array_equal(g[f], o[f], err_msg=f)
    np.testing.assert_array_equal(g["gap_hist"], o["gap_hist"])
    # one plain launch per interval gives the same answers
    for i in range(0, k, 9):
        s = gpu_ctx.sieve_intervals(lo[i:i + 1], hi[i:i + 1])
        for f in ("prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo"):
            assert s[f][0] == g[f][i]
        np.testing.assert_array_equal(s["gap_hist"][0], g["gap_hist"][i])


def test_primes_range_matches_oracle(gpu_ctx):
    for lo, hi in [(0, 100), (1, 10**6), (10**9, 10**9 + 3 * 10**6), (10**12 - 10**6, 10**12)]:
        g = gpu_ctx.primes_range(lo, hi)
        o = O.primes_range(lo, hi)
        np.testing.assert_array_equal(g, o)


def test_high_intervals_match_oracle(gpu_ctx_big):
    """Intervals up to 10^16 (base primes to 10^8): every prime category, including the
    multiples walk of primes larger than the tile's span."""
    rng = np.random.default_rng(20261203)
    k = 24
    lo = (np.floor(10 ** rng.uniform(10, 16, k) / 30) * 30).astype(np.uint64)
    ln = (10 ** rng.uniform(3, 6.3, k)).astype(np.uint64)
    lo[:3] = [10**16 - 10**6, 10**15, 3 * 10**15 + 7]
    hi = lo + ln
    g = gpu_ctx_big.sieve_intervals(lo, hi)
    o = O.sieve_intervals(lo, hi)
    for f in ("prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "gap_overflow"):
        np.testing.assert_array_equal(g[f], o[f], err_msg=f)
    np.testing.assert_array_equal(g["gap_hist"], o["gap_hist"])
    for i in (0, 1, 2):
        gr = gpu_ctx_big.sieve_range(int(lo[i]), int(hi[i]))
        orr = O.sieve_range(int(lo[i]), int(hi[i]))
        assert_range_equal(gr, orr)


def test_interval_near_1e18(gpu_ctx_big):
    lo, hi = 10**18 - 2 * 10**5, 10**18 + 10**5
    g = gpu_ctx_big.sieve_range(lo, hi)
    o = O.sieve_range(lo, hi)
    assert_range_equal(g, o)


def test_gaps_at_least_matches_oracle(gpu_ctx):
    for lo, hi, gmin in [(1, 10**7, 100), (10**9, 10**9 + 5 * 10**7, 150), (10**12 - 10**8, 10**12, 200)]:
        ps = O.primes_range(lo, hi).astype(np.int64)
        d = np.diff(ps)
        sel = np.nonzero(d >= gmin)[0]
        got = gpu_ctx.gaps_at_least(lo, hi, gmin)
        np.testing.assert_array_equal(got["position"], ps[sel + 1].astype(np.uint64))
        np.testing.assert_array_equal(got["gap"], d[sel].astype(np.int32))
        want_m = (d[sel] / np.log(ps[sel].astype(np.float64))).astype(np.float32)
        np.testing.assert_allclose(got["merit"], want_m, rtol=4e-6)


@pytest.mark.parametrize("compat", [True, False])
def test_sharded_ranges_merge_to_the_whole(gpu_ctx, compat):
    """The multi-GPU exchange of bench.py on one GPU: rank r sieves [r n + 1, (r+1) n + 1),
    its statistics struct travels as raw bytes (the NCCL all-gather payload), and
    voss_stats_merge adds the seam gaps; the result must equal one call over the whole range
    (reference-compat segment boundaries fall inside and between the shards)."""
    import voss
    from voss import _native as N
    world, n = 4, 10**10
    seg = SEG if compat else 0
    whole = gpu_ctx.sieve_range(1, world * n + 1, compat=compat, seg_num=seg, large_cap=1 << 20)
    shards = [gpu_ctx.sieve_range(r * n + 1, (r + 1) * n + 1, compat=compat, seg_num=seg, large_cap=1 << 20)
              for r in range(world)]
    # counts and histograms from the raw structs alone, as bench.py gathers them
    parts = [voss.range_result(N.RangeStats.from_buffer_copy(bytes(s.raw))) for s in shards]
    m = voss.merge_stats(parts)
    for k in ("prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "large_total"):
        assert getattr(m, k) == getattr(whole, k), k
    for k in ("mod4", "modq", "modq_gap", "gap_hist"):
        np.testing.assert_array_equal(getattr(m, k), getattr(whole, k), err_msg=k)
    # with the large-gap lists as well
    m2 = voss.merge_stats(shards)
    assert sorted(zip(m2.large["position"].tolist(), m2.large["gap"].tolist())) == \
        sorted(zip(whole.large["position"].tolist(), whole.large["gap"].tolist()))


def _same_intervals(a, b):
    for f in ("lo", "hi", "prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "gap_overflow"):
        np.testing.assert_array_equal(a[f], b[f], err_msg=f)
    np.testing.assert_array_equal(a["gap_hist"], b["gap_hist"])


def test_short_intervals_by_miller_rabin_equal_the_sieve(gpu_ctx_big):
    """Short intervals at high starts go to the Miller-Rabin path (short_iv.cu); with the route
    switched off the same batch is sieved.  Both must agree bit for bit, for a mixed batch, a
    batch routed entirely, intervals without wheel integers, and against the oracle."""
    rng = np.random.default_rng(11)
    k = 96
    lo = (10 ** rng.uniform(9, 18, k)).astype(np.uint64)
    ln = (10 ** rng.uniform(0, 6, k)).astype(np.uint64)
    base = 30 * (10**16 // 30)
    lo[:4] = [base + 2, base + 1, 10**18 - 10**4, 3 * 10**17 + 11]
    ln[:4] = [5, 1, 10**4, 3]                       # no wheel integer; only base + 1; ...
    hi = lo + ln
    t0 = gpu_ctx_big.tuning()
    try:
        routed = gpu_ctx_big.sieve_intervals(lo, hi)
        gpu_ctx_big.set_tuning(**{**t0, "mr_route": 0xFFFFFFFF})
        sieved = gpu_ctx_big.sieve_intervals(lo, hi)
        _same_intervals(routed, sieved)
        gpu_ctx_big.set_tuning(**t0)
        only = gpu_ctx_big.sieve_intervals(lo[:4], hi[:4])      # every interval routed: no sieve launch
        assert gpu_ctx_big.last_phase_ms()[3] == 4              # candidates, two Miller-Rabin kernels, statistics
        _same_intervals(only, sieved[:4])
    finally:
        gpu_ctx_big.set_tuning(**t0)
    sel = np.nonzero(hi < 10**16)[0][:16]
    _same_intervals(routed[sel], O.sieve_intervals(lo[sel], hi[sel]))


def test_large_interval_batches_through_staging(gpu_ctx):
    """Batches whose results exceed 8 MB (over 1023 intervals) come back through the context's
    pinned staging; they equal the same intervals in small batches and the oracle."""
    rng = np.random.default_rng(23)
    k = 2500
    lo = (10 ** rng.uniform(1, 12.5, k)).astype(np.uint64)
    hi = lo + (10 ** rng.uniform(0, 4, k)).astype(np.uint64)
    big = gpu_ctx.sieve_intervals(lo, hi)
    small = np.concatenate([gpu_ctx.sieve_intervals(lo[i:i + 500], hi[i:i + 500]) for i in range(0, k, 500)])
    _same_intervals(big, small)
    sel = np.arange(0, k, 37)
    _same_intervals(big[sel], O.sieve_intervals(lo[sel], hi[sel]))


def test_intervals_at_the_top_of_the_supported_range():
    """Intervals just below 2^62 (the largest max_hi a context takes): base primes up to 2^31,
    so the large-prime pre-pass meets primes of 2^30 and more, whose remainders take its 64-bit
    form.  Sieved (Miller-Rabin route off) and routed, both equal to the oracle."""
    import voss
    top = 1 << 62
    lo = np.array([top - 10**6, top - 3 * 10**5 - 17, top - 2 * 10**7], dtype=np.uint64)
    hi = np.array([top, top - 10**5, top - 2 * 10**7 + 4 * 10**5], dtype=np.uint64)
    want = O.sieve_intervals(lo, hi)
    with voss.Context(top) as ctx:
        t0 = ctx.tuning()
        routed = ctx.sieve_intervals(lo, hi)
        ctx.set_tuning(**{**t0, "mr_route": 0xFFFFFFFF})
        sieved = ctx.sieve_intervals(lo, hi)
    _same_intervals(sieved, want)
    _same_intervals(routed, want)

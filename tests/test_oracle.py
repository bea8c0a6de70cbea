"""Pins the CPU oracle (oracle/liboracle.so) to the reference's known answers and to the
reference verifier compiled unmodified (oracle/_ref/libref_verify.so).  CPU only."""
import json
import math
import os

import numpy as np
import pytest

import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
SEG = 30_000_000_000


def brute_primes(n):
    s = np.ones(n + 1, dtype=bool)
    s[:2] = False
    for i in range(2, int(n**0.5) + 1):
        if s[i]:
            s[i * i::i] = False
    return np.nonzero(s)[0].astype(np.uint64)


def brute_stats(lo, hi, compat, seg):
    """Pure-Python statement of the reference's per-pair rules (voss_v7_live.cu:278-299,
    :551-562, :634-635, :682), for small ranges."""
    ps = [int(p) for p in brute_primes(max(hi, 2)) if lo <= p < hi]
    W = [1, 7, 11, 13, 17, 19, 23, 29]
    hist, modq_gap, large = {}, {}, []
    mod4 = [0, 0]
    for p in ps:
        if p % 4 == 1:
            mod4[0] += 1
        elif p % 4 == 3:
            mod4[1] += 1
    max_gap, max_lo = 0, 0
    for a, b in zip(ps, ps[1:]):
        g = b - a
        hist[g] = hist.get(g, 0) + 1
        if g > max_gap:
            max_gap, max_lo = g, a
        if a < 7 or (compat and (a - 1) // seg != (b - 1) // seg):
            continue
        if g < 100:
            r6 = 0 if a % 6 == 1 else 1
            modq_gap[(r6, g)] = modq_gap.get((r6, g), 0) + 1
            r30 = 2 + W.index(a % 30)
            modq_gap[(r30, g)] = modq_gap.get((r30, g), 0) + 1
        merit = g / math.log(a) if g > 100 else 0.0
        if g >= 500 or merit >= 10.0:
            large.append((b, g))
    return dict(count=len(ps), hist=hist, modq_gap=modq_gap, large=large, mod4=mod4, max_gap=max_gap,
                max_lo=max_lo, first=ps[0] if ps else 0, last=ps[-1] if ps else 0)


@pytest.mark.parametrize("n", range(1, 10))
def test_pi_10n(n):
    r = O.sieve_range(1, 10**n + 1, compat=True, seg_num=SEG)
    assert r.prime_count == GOLD["pi_10n"][str(n)]
    # the reference's three self-checks (voss_v7_live.cu:693-705)
    gh = r.gap_hist
    assert int(gh.sum()) == r.prime_count - 1
    assert int((np.arange(gh.size, dtype=np.uint64) * gh).sum()) == r.last_prime - 2
    assert int(r.mod4.sum()) + 1 == r.prime_count


def test_hist_1000_and_chebyshev_1e9():
    r = O.sieve_range(1, 1001, compat=True, seg_num=SEG)
    assert {str(g): int(c) for g, c in enumerate(r.gap_hist) if c} == GOLD["gap_hist"]["1000"]
    r = O.sieve_range(1, 10**9 + 1, compat=True, seg_num=SEG)
    assert [int(r.mod4[0]), int(r.mod4[1])] == GOLD["chebyshev"][str(10**9)]
    assert (r.max_gap, r.max_gap_lo) == (282, 436273009)  # the maximal gap below 1e9


def test_sieve_work_matches_baseline_table():
    assert O.sieve_work(10**9) == 404309576
    assert O.sieve_work(10**12) == 484385202990


def test_bench_sieve_work_equals_oracle():
    """bench.py's roofline counts H(n) with its own numpy statement; it must equal the
    oracle's count, including the difference form used for a rank's sub-range."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for n in (1, 48, 49, 50, 10**6 + 7, 10**9, 2 * 10**12, 10**12):
        assert bench.sieve_work(n) == O.sieve_work(n), n


def _bench():
    import importlib.util
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def test_bench_interval_work_terms():
    """The interval roofline's work terms: the offsets are exact (one per interval and base
    prime <= isqrt(hi - 1)); the expected clear counts agree with a direct count of the wheel
    multiples of each prime (>= p^2) within a few per cent on intervals of 10^6."""
    bench = _bench()
    lo = np.array([10**8, 10**10, 3 * 10**11], dtype=np.uint64)
    hi = lo + np.array([10**6, 10**6, 10**6], dtype=np.uint64)
    p_large = 20_000
    w = bench.interval_work(lo, hi, p_large)
    P = bench.primes_upto(math.isqrt(int(hi.max()) - 1)).astype(np.int64)
    assert w["first_hit_offsets"] == sum(int((P <= math.isqrt(int(h) - 1)).sum()) for h in hi)
    exact = [0, 0, 0]
    cuts = [7, 37, p_large, 1 << 62]
    for a, b in zip(lo.tolist(), hi.tolist()):
        for p in P[P <= math.isqrt(b - 1)].tolist():
            m0 = max(-(-a // p), p)            # first multiple >= max(a, p^2), as a multiplier
            m1 = (b - 1) // p
            if m1 < m0:
                continue
            def coprime_upto(x):               # multipliers m <= x coprime to 30
                return 8 * (x // 30) + sum(1 for r in range(1, x % 30 + 1) if math.gcd(r, 30) == 1)
            c = coprime_upto(m1) - coprime_upto(m0 - 1)
            exact[next(i for i in range(3) if cuts[i] <= p < cuts[i + 1])] += c
    got = [w["presieve_primes_hits"], w["tile_hits"], w["prepass_hits"]]
    for g, e in zip(got, exact):
        assert abs(g - e) <= 0.03 * e + 50, (got, exact)


def test_bench_mr_products_small_cases():
    """The Miller-Rabin roofline's product count for single candidates, by hand."""
    bench = _bench()
    assert bench.mr_mulmods(np.array([2, 3, 4, 9, 35, 37], dtype=np.uint64)) == (0, 0)  # trial division
    # 41: d = 5 (3 bits, 2 set), r = 3; base 2: 3 squarings, 2^5 = 32 = -9, squarings to -1:
    # 32^2 = 40 = -1 after one step.  Bases 3, 5, 7, 11, 13: 3 + 2 products each plus the steps.
    n = 41
    want = 0
    for a in (2, 3, 5, 7, 11, 13):
        want += 3 + (0 if a == 2 else 2)
        x = pow(a, 5, n)
        j = 0
        while x not in (1, n - 1) and j < 2:
            x = x * x % n
            j += 1
        want += j
    assert bench.mr_mulmods(np.array([n], dtype=np.uint64)) == (want, 0)
    big = (1 << 63) + 29                       # above 2^63: counted as a full-width modulus
    s, f = bench.mr_mulmods(np.array([big], dtype=np.uint64))
    assert s == 0 and f > 0


@pytest.mark.parametrize("n,span", [(10**12, 4 * 10**9), (10**12, 10**8), (10**9, 10**9), (1000, 5000), (100, 7)])
def test_bench_cpu_sample_is_stratified_over_the_range(n, span):
    """The CPU baseline's sample: 8 equal slices inside [1, n + 1), one centred in each eighth."""
    bench = _bench()
    sl = bench.sample_slices(n, span)
    assert len(sl) == 8
    widths = {hi - lo for lo, hi in sl}
    assert len(widths) == 1 and widths.pop() == max(1, span // 8)
    for j, (lo, hi) in enumerate(sl):
        assert 1 <= lo < hi <= n + 1
        if span // 8 <= n // 8:  # a slice fits its eighth: it lies around the eighth's middle
            assert lo <= 1 + (2 * j + 1) * n // 16 < hi or hi - lo == 1
    assert [lo for lo, _ in sl] == sorted(lo for lo, _ in sl)


@pytest.mark.parametrize("lo,hi,compat,seg", [
    (1, 20000, True, 30), (1, 20000, True, 330), (1, 50000, True, 30_000_000_000),
    (1, 20000, False, 0), (2, 3, False, 0), (0, 8, False, 0), (9000, 31000, False, 0),
    (9000, 31000, True, 990),
])
def test_oracle_against_python_statement(lo, hi, compat, seg):
    r = O.sieve_range(lo, hi, compat=compat, seg_num=seg)
    b = brute_stats(lo, hi, compat, seg)
    assert r.prime_count == b["count"]
    assert (r.first_prime, r.last_prime) == (b["first"], b["last"])
    assert (r.max_gap, r.max_gap_lo) == (b["max_gap"], b["max_lo"])
    assert {g: int(c) for g, c in enumerate(r.gap_hist) if c} == b["hist"]
    got_mg = {(i, g): int(r.modq_gap[i, g]) for i in range(10) for g in range(100) if r.modq_gap[i, g]}
    assert got_mg == b["modq_gap"]
    assert sorted(zip(r.large["position"].tolist(), r.large["gap"].tolist())) == sorted(b["large"])
    assert list(map(int, r.mod4)) == b["mod4"]


def test_oracle_modq_counts_small():
    lo, hi = 1, 30001
    r = O.sieve_range(lo, hi)
    ps = brute_primes(hi - 1)
    for q in (3, 4, 5, 6, 7, 8, 11, 12, 13, 30):
        want = np.bincount((ps % q).astype(np.int64), minlength=q)
        np.testing.assert_array_equal(r.modq_counts(q), want)


def test_oracle_intervals_and_primes():
    lo = np.array([0, 1, 2, 100, 10**6, 999_983], dtype=np.uint64)
    hi = np.array([10, 2, 100, 10**5, 10**6 + 10**4, 999_984], dtype=np.uint64)
    out = O.sieve_intervals(lo, hi)
    for i in range(lo.size):
        ps = [int(p) for p in brute_primes(int(hi[i]) + 1) if lo[i] <= p < hi[i]]
        assert out["prime_count"][i] == len(ps)
        gaps = np.diff(np.array(ps, dtype=np.int64))
        want = np.zeros(1024, dtype=np.uint64)
        for g in gaps:
            want[g >> 1] += 1
        np.testing.assert_array_equal(out["gap_hist"][i], want)
        np.testing.assert_array_equal(O.primes_range(int(lo[i]), int(hi[i])), np.array(ps, dtype=np.uint64))


def test_oracle_long_intervals_split_into_chunks():
    """Intervals longer than the oracle's 2^24-integer chunk are sieved chunk by chunk in
    parallel and merged with the gaps across the seams: the statistics equal the range
    oracle's (one accumulator per thread span) and pi(10^9) from the reference's table."""
    lo = np.array([0, 10**9 - 3 * 2**24 - 5, 10**12 - 5 * 10**7], dtype=np.uint64)
    hi = np.array([10**9, 10**9 + 2**24 + 11, 10**12 + 7], dtype=np.uint64)
    out = O.sieve_intervals(lo, hi)
    assert out["prime_count"][0] == 50_847_534
    for i in range(lo.size):
        r = O.sieve_range(int(lo[i]), int(hi[i]))
        assert out["prime_count"][i] == r.prime_count
        assert (out["first_prime"][i], out["last_prime"][i]) == (r.first_prime, r.last_prime)
        assert (out["max_gap"][i], out["max_gap_lo"][i]) == (r.max_gap, r.max_gap_lo)
        want = np.zeros(1024, dtype=np.uint64)
        for g, c in enumerate(r.gap_hist):
            if c:
                want[g >> 1] += c
        np.testing.assert_array_equal(out["gap_hist"][i], want)


needs_ref = pytest.mark.skipif(not os.path.exists(O.REF_VERIFY_SO),
                               reason="oracle/_ref/libref_verify.so not built (reference tree absent)")

SPECIAL = [0, 1, 2, 3, 4, 5, 9, 25, 37, 41, 1369, 2047, 3215031751, 341550071728321, 3825123056546413051,
           18446744073709551557, 18446744073709551615, 2**61 - 1, 4759123141, 1122004669633]


@needs_ref
def test_mr_port_matches_reference_verifier():
    rng = np.random.default_rng(5)
    n = np.concatenate([np.array(SPECIAL, dtype=np.uint64),
                        rng.integers(0, 2**63, 200_000, dtype=np.uint64) * 2 + 1,
                        rng.integers(0, 10**6, 50_000, dtype=np.uint64),
                        brute_primes(200_000)])
    np.testing.assert_array_equal(O.mr_batch(n), O.ref_mr_batch(n))


@needs_ref
def test_prove_gaps_port_matches_reference_verifier():
    r = O.sieve_range(1, 10**8 + 1, compat=True, seg_num=SEG)
    p = r.large["position"].astype(np.uint64)
    g = r.large["gap"].astype(np.int32)
    P = np.concatenate([p, p[:40] + 2, np.array([3, 5, 7, 11, 13, 2, 29, 97, 1009, 5], dtype=np.uint64)])
    G = np.concatenate([g, g[:40], np.array([1, 3, 4, 2, 2, 0, -3, 8, 1006, 2], dtype=np.int32)])
    want = O.ref_prove_gaps(P, G)
    np.testing.assert_array_equal(O.prove_gaps(P, G), want)
    assert want[: p.size].all()

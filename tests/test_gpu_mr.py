"""GPU Miller-Rabin and gap proofs against the reference verifier compiled unmodified
(oracle/_ref/libref_verify.so) and the oracle restatement.  Exact (bool) comparison."""
import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

SPECIAL = [0, 1, 2, 3, 4, 5, 9, 25, 37, 41, 43, 1369, 2047, 3215031751, 341550071728321,
           3825123056546413051, 18446744073709551557, 18446744073709551615, 18446744073709551614,
           2**61 - 1, 2**63 - 25, 2**64 - 59, 1000000007, 999999999989, 4759123141, 1122004669633,
           # smallest strong pseudoprimes to the first 2, 3, 5, 6 prime bases (OEIS A014233)
           1373653, 25326001, 2152302898747, 3474749660383, 3474749660383 + 2, 341550071728321 - 2]


def checker(n):
    import os
    if os.path.exists(O.REF_VERIFY_SO):
        return O.ref_mr_batch(n)
    return O.mr_batch(n)


def test_mr_special_values(gpu_ctx):
    n = np.array(SPECIAL, dtype=np.uint64)
    np.testing.assert_array_equal(gpu_ctx.mr_verify(n), checker(n))


def test_mr_random_odd_and_primes(gpu_ctx):
    rng = np.random.default_rng(20261203)
    r = rng.integers(0, 2**63, size=200_000, dtype=np.uint64) * 2 + 1
    p = gpu_ctx.primes_range(10**12 - 3 * 10**6, 10**12)
    n = np.concatenate([r, p, p + 2, (p[:1000] * p[1:1001]).astype(np.uint64)])
    got = gpu_ctx.mr_verify(n)
    np.testing.assert_array_equal(got, checker(n))
    assert got[r.size:r.size + p.size].all()


def test_mr_strong_pseudoprimes(gpu_ctx):
    # products of two primes p*(2p-1) style values that pass a few bases
    rng = np.random.default_rng(1)
    q = gpu_ctx.primes_range(10**6, 2 * 10**6)
    a = rng.choice(q, 5000)
    b = 2 * a - 1
    n = (a * b).astype(np.uint64)
    np.testing.assert_array_equal(gpu_ctx.mr_verify(n), checker(n))


def test_mr_bands_of_base_counts(gpu_ctx):
    """Random odd values in each band where a different number of bases is exact (below
    3,474,749,660,383: 6; below 341,550,071,728,321: 7; below 3,825,123,056,546,413,051: 9;
    above: 12), the bands' edges, and sieved primes on both sides of the first edge."""
    rng = np.random.default_rng(77)
    edges = [3474749660383, 341550071728321, 3825123056546413051]
    lo_hi = [(10**6, edges[0]), (edges[0], edges[1]), (edges[1], edges[2]), (edges[2], 2**64 - 1)]
    parts = [(rng.integers(a // 2, b // 2, 100_000, dtype=np.uint64) * 2 + 1) for a, b in lo_hi]
    parts.append(np.array([e + d for e in edges for d in range(-41, 42, 2)], dtype=np.uint64))
    parts.append(gpu_ctx.primes_range(edges[0] - 3 * 10**5, edges[0] + 3 * 10**5))
    n = np.concatenate(parts)
    np.testing.assert_array_equal(gpu_ctx.mr_verify(n), checker(n))


def test_prove_gaps(gpu_ctx):
    r = gpu_ctx.sieve_range(1, 10**10 + 1, compat=True)
    lg = r.large
    p = lg["position"].astype(np.uint64)
    g = lg["gap"].astype(np.int32)
    # corrupt some: wrong gap, non-prime end, gap 1/0/negative, p_before = 2 cases
    bad_p = np.concatenate([p[:50], p[:50] + 2, np.array([3, 5, 7, 11, 13, 2, 29, 97], dtype=np.uint64)])
    bad_g = np.concatenate([g[:50] - 2, g[:50], np.array([1, 3, 4, 2, 2, 0, -3, 8], dtype=np.int32)])
    P = np.concatenate([p, bad_p])
    G = np.concatenate([g, bad_g])
    got = gpu_ctx.prove_gaps(P, G)
    want = O.ref_prove_gaps(P, G) if __import__("os").path.exists(O.REF_VERIFY_SO) else O.prove_gaps(P, G)
    np.testing.assert_array_equal(got, want)
    assert got[: p.size].all()


def test_prove_gaps_long_joined_and_high(gpu_ctx):
    """Proofs that span several 256-integer rounds (the maximal gap below 1e12, found by the
    sieve), joined gaps whose interior holds a prime, and endpoints just below 2^64."""
    checker = O.ref_prove_gaps if __import__("os").path.exists(O.REF_VERIFY_SO) else O.prove_gaps
    big = gpu_ctx.gaps_at_least(7 * 10**11, 8 * 10**11, 500)
    assert big.size and int(big["gap"].max()) >= 514
    ps = gpu_ctx.primes_range(10**11, 10**11 + 20000)
    joined_p = ps[2:200]
    joined_g = (ps[2:200] - ps[:198]).astype(np.int32)  # interior holds ps[1:199]
    odd = np.uint64(2**64 - 3001) + np.arange(0, 3000, 2, dtype=np.uint64)
    top = odd[gpu_ctx.mr_verify(odd).astype(bool)]
    assert top.size >= 3
    top_p, top_g = top[1:], (top[1:] - top[:-1]).astype(np.int32)
    P = np.concatenate([big["position"].astype(np.uint64), joined_p, top_p, top_p[:1]])
    G = np.concatenate([big["gap"].astype(np.int32), joined_g, top_g, 2 * top_g[:1]])  # last: holds top[0] or starts at a composite
    got = gpu_ctx.prove_gaps(P, G)
    nb, nj = big.size, joined_p.size
    # the reference checker sieves with every prime below isqrt(p_after): affordable below 1e12;
    # near 2^64 every odd integer of the window was tested above, so consecutive entries of
    # `top` are consecutive primes and their proofs must hold
    np.testing.assert_array_equal(got[:nb + nj], checker(P[:nb + nj], G[:nb + nj]))
    assert got[:nb].all() and not got[nb:nb + nj].any()
    assert got[nb + nj:-1].all() and not got[-1]


def test_mr_large_host_batches_through_staging(gpu_ctx):
    """Batches of 2^20 candidates or more cross through the context's pinned staging buffers
    (one and several 2^24-candidate chunks, odd sizes); their verdicts equal those of small
    batches, which are copied straight from the caller's memory, and the reference verifier's."""
    rng = np.random.default_rng(5)
    for size in (3 * 2**20 + 7, 2**24 + 12345):
        n = rng.integers(0, 2**63, size=size, dtype=np.uint64) * 2 + 1
        n[::97] = rng.integers(0, 2**40, size=n[::97].size, dtype=np.uint64)  # even and small values too
        got = gpu_ctx.mr_verify(n)
        step = (1 << 20) - 1
        small = np.concatenate([gpu_ctx.mr_verify(n[i:i + step]) for i in range(0, size, step)])
        np.testing.assert_array_equal(got, small)
        sel = np.arange(0, size, 53)
        np.testing.assert_array_equal(got[sel], checker(n[sel]))


def test_prove_gaps_large_batches_through_staging(gpu_ctx):
    """2^20 gaps or more cross through the pinned staging buffers; the verdicts (true gaps and
    altered ones) equal those of small batches and of the reference verifier on a sample."""
    gaps = gpu_ctx.gaps_at_least(1, 5 * 10**9, 100)
    assert gaps.size > (1 << 20)
    p = gaps["position"].astype(np.uint64)
    g = gaps["gap"].astype(np.int32)
    g[::11] += 2                                   # a larger gap whose interior holds a prime
    got = gpu_ctx.prove_gaps(p, g)
    step = (1 << 20) - 1
    small = np.concatenate([gpu_ctx.prove_gaps(p[i:i + step], g[i:i + step]) for i in range(0, p.size, step)])
    np.testing.assert_array_equal(got, small)
    assert got[1::11].all() and not got[::11].any()
    import os
    sel = np.arange(0, p.size, 997)
    ref = O.ref_prove_gaps(p[sel], g[sel]) if os.path.exists(O.REF_VERIFY_SO) else O.prove_gaps(p[sel], g[sel])
    np.testing.assert_array_equal(got[sel], ref)


def test_staging_in_many_chunks_equals_direct_copies(monkeypatch):
    """With the staging buffers limited to 2^17 entries (VOSS_STAGE_LIMIT, read when a context is
    created) every staged transfer crosses in many chunks that alternate between the two
    buffers: Miller-Rabin candidates in and verdicts out, gap proofs in and out, and interval
    results out.  Each result equals the same work in batches small enough to be copied
    directly."""
    import voss
    monkeypatch.setenv("VOSS_STAGE_LIMIT", str(1 << 17))
    rng = np.random.default_rng(31)
    with voss.Context(10**12) as ctx:
        n = rng.integers(0, 2**63, size=3 * 2**20 + 5, dtype=np.uint64) * 2 + 1
        n[::89] = rng.integers(0, 10**9, size=n[::89].size, dtype=np.uint64)
        got = ctx.mr_verify(n)
        step = (1 << 20) - 1
        np.testing.assert_array_equal(got, np.concatenate([ctx.mr_verify(n[i:i + step])
                                                           for i in range(0, n.size, step)]))
        sel = np.arange(0, n.size, 101)
        np.testing.assert_array_equal(got[sel], checker(n[sel]))
        gaps = ctx.gaps_at_least(1, 3 * 10**9, 90)
        assert gaps.size > (1 << 20)
        p = gaps["position"].astype(np.uint64)
        g = gaps["gap"].astype(np.int32)
        g[::7] += 2
        ok = ctx.prove_gaps(p, g)
        np.testing.assert_array_equal(ok, np.concatenate([ctx.prove_gaps(p[i:i + step], g[i:i + step])
                                                          for i in range(0, p.size, step)]))
        assert not ok[::7].any() and ok[1::7].all()
        lo = (10 ** rng.uniform(3, 11, 1500)).astype(np.uint64)
        hi = lo + (10 ** rng.uniform(0, 4, lo.size)).astype(np.uint64)
        big = ctx.sieve_intervals(lo, hi)                 # 12 MB of results: staged, 12 chunks
        small = np.concatenate([ctx.sieve_intervals(lo[i:i + 500], hi[i:i + 500]) for i in range(0, lo.size, 500)])
        for f in voss.INTERVAL_DTYPE.names:
            np.testing.assert_array_equal(big[f], small[f], err_msg=f)

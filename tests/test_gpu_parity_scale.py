"""Oracle parity at the benchmark workloads' own magnitudes.

The batched-interval benchmark (4096 seeded intervals, starts to 10^16, lengths to 10^8), the
serving benchmark's request stream (starts to 10^18, lengths to 10^9, Miller-Rabin batches of
10^3..10^6 odd values) and the verification benchmark (10^8 candidates, gap proofs of every gap
>= 200 below 10^12) are checked here against the CPU oracle, which restates the reference's
interval marking loop (src/verify_cpp.cpp:73-90), and against the reference verifier compiled
unmodified (src/verify_cpp.cpp:24-93).  The GPU runs each workload whole, exactly as the
benchmark does; the CPU checks a seeded sample that always includes the longest intervals and
the highest starts.  Integer work: every comparison is exact.
"""
import os
import sys

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402  (interval_batch, mr_candidates: the benchmark's own inputs)

SEED = 20261203
FIELDS = ("lo", "hi", "prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "gap_overflow")


def _same_intervals(g, o, what):
    for f in FIELDS:
        np.testing.assert_array_equal(g[f], o[f], err_msg=f"{what}: {f}")
    np.testing.assert_array_equal(g["gap_hist"], o["gap_hist"], err_msg=f"{what}: gap_hist")


def _mr_checker(n):
    return O.ref_mr_batch(n) if os.path.exists(O.REF_VERIFY_SO) else O.mr_batch(n)


def test_interval_benchmark_batch_matches_oracle():
    """All 4096 intervals in one batched launch on a context sized as the benchmark's (base
    primes to 10^8); 56 of them against the oracle: the 8 longest (L near 10^8), the 8 highest
    starts (near 10^16) and 40 drawn with a fixed seed."""
    import voss
    lo, hi = bench.interval_batch(4096, SEED)
    with voss.Context(int(hi.max()) + 1) as ctx:
        got = ctx.sieve_intervals(lo, hi)
    span = hi - lo
    longest = np.argsort(span)[-8:]
    highest = np.argsort(lo)[-8:]
    rng = np.random.default_rng(5)
    rest = rng.choice(np.setdiff1d(np.arange(lo.size), np.concatenate([longest, highest])), 40, replace=False)
    sel = np.unique(np.concatenate([longest, highest, rest]))
    assert span[sel].max() > 9 * 10**7 and lo[sel].max() > 9 * 10**15
    _same_intervals(got[sel], O.sieve_intervals(lo[sel], hi[sel]), "4096-interval batch")


def test_serving_stream_through_the_server_matches_oracle(gpu_ctx_big):
    """The serving benchmark's 10^3 req/s stream (default magnitudes).  Its requests go through
    the continuous-batching server as fast as they can be submitted, so they share batches and
    overlap; a sample of the interval requests is checked against the oracle (the highest
    starts, near 10^18, with lengths up to 10^7; the longest, near 10^9; 20 drawn with a fixed
    seed) and a sample of the Miller-Rabin requests against the reference verifier."""
    from voss.serve import Server, request_stream
    stream = request_stream(1e3, 3000, seed=SEED)
    iv = [i for i, (_, k, _) in enumerate(stream) if k == "iv"]
    mr = [i for i, (_, k, _) in enumerate(stream) if k == "mr"]
    lo = np.array([stream[i][2][0] for i in iv], dtype=np.uint64)
    hi = np.array([stream[i][2][1] for i in iv], dtype=np.uint64)
    span = hi - lo
    by_start = [j for j in np.argsort(lo)[::-1] if span[j] <= 10**7][:6]
    by_len = [j for j in np.argsort(span)[::-1] if lo[j] < 10**13][:3]
    rng = np.random.default_rng(3)
    pool = np.setdiff1d(np.nonzero(span <= 10**7)[0], by_start)
    sel = np.unique(np.concatenate([by_start, by_len, rng.choice(pool, 20, replace=False)]))
    assert lo[sel].max() > 9 * 10**17 and span[sel].max() > 5 * 10**8
    mr_sel = sorted(rng.choice(mr, 40, replace=False).tolist())
    # submit in arrival order: the sampled intervals and Miller-Rabin batches, plus every other
    # interval request shorter than 10^6 so the batches are mixed
    wanted = set(iv[j] for j in sel) | set(mr_sel)
    order = [i for i in range(len(stream))
             if i in wanted or (stream[i][1] == "iv" and stream[i][2][1] - stream[i][2][0] < 10**6)]
    tickets = {}
    with Server(gpu_ctx_big, slots=4) as srv:
        for i in order:
            _, kind, payload = stream[i]
            tickets[i] = srv.submit_interval(*payload) if kind == "iv" else srv.submit_mr(payload)[0]
        got_iv, got_mr = {}, {}
        for i in order:
            assert srv.wait(tickets[i], 600_000) == 0, i
            if i in wanted:
                kind, payload = stream[i][1], stream[i][2]
                if kind == "iv":
                    got_iv[i] = srv.result_interval(tickets[i])
                else:
                    got_mr[i] = srv.result_mr(tickets[i], payload.size)
            srv.release(tickets[i])
        st = srv.stats()
    assert st["failed"] == 0 and st["batches"] < len(order)
    g = np.array([got_iv[iv[j]] for j in sel], dtype=got_iv[iv[sel[0]]].dtype)
    _same_intervals(g, O.sieve_intervals(lo[sel], hi[sel]), "served intervals")
    for i in mr_sel:
        np.testing.assert_array_equal(got_mr[i], _mr_checker(stream[i][2]), err_msg=f"request {i}")


def test_verification_benchmark_batch_matches_reference(gpu_ctx):
    """The 10^8-candidate Miller-Rabin batch (5*10^7 primes below 10^12 + 5*10^7 random odd
    u64) verified whole on the device; 4*10^6 seeded positions against the reference's
    is_prime_u64, every known prime reported prime.  Then every gap >= 200 below 10^12 is
    proved on the device and 20,000 of them against the reference's verify_gap."""
    n, known = bench.mr_candidates(gpu_ctx, 50_000_000, SEED)
    assert n.size == 10**8
    got = gpu_ctx.mr_verify(n)
    assert got[known].all()
    rng = np.random.default_rng(9)
    sample = np.sort(rng.choice(n.size, 4_000_000, replace=False))
    np.testing.assert_array_equal(got[sample], _mr_checker(n[sample]))
    gaps = gpu_ctx.gaps_at_least(1, 10**12 + 1, 200)
    assert gaps.size == 8_044_902  # results/hist_snapshots/hist_1000000000000.csv, gaps >= 200
    p_after = gaps["position"].astype(np.uint64)
    g = gaps["gap"].astype(np.int32)
    ok = gpu_ctx.prove_gaps(p_after, g)
    assert ok.all()
    ps = np.sort(rng.choice(p_after.size, 20_000, replace=False))
    want = O.ref_prove_gaps(p_after[ps], g[ps]) if os.path.exists(O.REF_VERIFY_SO) else O.prove_gaps(p_after[ps], g[ps])
    np.testing.assert_array_equal(ok[ps], want)

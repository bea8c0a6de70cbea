"""The request server: continuous batching must not change any answer.  Each result served in a
mixed, overlapping stream equals the same request served alone (one plain call); failures
injected on the host fail only their own batch; every wait is bounded."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mixed_requests(seed, count):
    from voss.serve import request_stream
    # magnitudes kept moderate so the comparison calls stay quick
    return request_stream(rate=1e4, count=count, seed=seed, start_exp=(1.0, 15.5), len_exp=(0.0, 7.0), mr_exp=(0.0, 4.5))


def test_results_same_alone_and_in_the_mix(gpu_ctx_big):
    import voss
    from voss.serve import Server
    reqs = mixed_requests(11, 400)
    tickets = [None] * len(reqs)
    with Server(gpu_ctx_big, slots=3, max_batch_requests=64) as srv:
        # two client threads submit interleaved, as fast as they can
        def submit(part):
            for i in part:
                _, kind, payload = reqs[i]
                tickets[i] = srv.submit_interval(*payload) if kind == "iv" else srv.submit_mr(payload)[0]
        ths = [threading.Thread(target=submit, args=(range(k, len(reqs), 2),)) for k in (0, 1)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        got = []
        for i, (_, kind, payload) in enumerate(reqs):
            assert srv.wait(tickets[i], 120_000) == 0
            got.append(srv.result_interval(tickets[i]) if kind == "iv" else srv.result_mr(tickets[i], payload.size))
            srv.release(tickets[i])
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] < len(reqs)  # requests were batched
    for (_, kind, payload), g in zip(reqs, got):
        if kind == "iv":
            alone = gpu_ctx_big.sieve_intervals(np.array([payload[0]], dtype=np.uint64),
                                                np.array([payload[1]], dtype=np.uint64))[0]
            for f in voss.INTERVAL_DTYPE.names:
                assert np.array_equal(g[f], alone[f]), (payload, f)
        else:
            np.testing.assert_array_equal(g, gpu_ctx_big.mr_verify(payload))


def test_injected_batch_failures_are_contained(gpu_ctx):
    from voss.serve import Server
    with Server(gpu_ctx, slots=1, max_batch_requests=4, fail_every_n_batches=3) as srv:
        tks = []
        for i in range(40):
            lo = 10**9 + i * 10**6
            tks.append((srv.submit_interval(lo, lo + 10**5), lo))
        rcs = [srv.wait(t, 60_000) for t, _ in tks]
        ok = [i for i, rc in enumerate(rcs) if rc == 0]
        bad = [i for i, rc in enumerate(rcs) if rc != 0]
        assert bad and ok
        assert all(rcs[i] == -2 for i in bad)  # VOSS_ERR_CUDA from the injected failure
        for i in ok:
            t, lo = tks[i]
            r = srv.result_interval(t)
            alone = gpu_ctx.sieve_intervals(np.array([lo], dtype=np.uint64), np.array([lo + 10**5], dtype=np.uint64))[0]
            assert r["prime_count"] == alone["prime_count"]
        st = srv.stats()
        assert st["failed"] == len(bad) and st["completed"] == len(ok)
        # the server keeps serving after failures
        t = srv.submit_interval(1, 1000)
        rc = srv.wait(t, 60_000)
        assert rc in (0, -2)


def test_bounded_wait_and_capacity_checks(gpu_ctx):
    import voss
    from voss.serve import Server
    with Server(gpu_ctx, slots=2, max_batch_tiles=8, max_batch_candidates=1000) as srv:
        with pytest.raises(voss.VossError) as e:
            srv.submit_interval(1, 10**11)      # needs more than 8 tiles
        assert e.value.code == -4
        with pytest.raises(voss.VossError):
            srv.submit_mr(np.arange(1001, dtype=np.uint64))
        t = srv.submit_interval(10**12, 10**12 + 10**7)
        rc = srv.wait(t, 0)                      # a zero timeout returns at once
        assert rc in (0, -6)
        assert srv.wait(t, 60_000) == 0
        with pytest.raises(voss.VossError):
            srv.release(123456789)


def test_batches_overlap_under_load(gpu_ctx):
    from voss.serve import Server
    with Server(gpu_ctx, slots=4, max_batch_requests=8) as srv:
        tks = [srv.submit_interval(10**12 + i * 10**8, 10**12 + (i + 1) * 10**8) for i in range(64)]
        assert all(srv.wait(t, 120_000) == 0 for t in tks)
        st = srv.stats()
    assert st["max_inflight_batches"] >= 2

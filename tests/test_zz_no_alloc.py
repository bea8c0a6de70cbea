"""voss_mr_verify_noalloc: Miller-Rabin for callers that cannot allocate device memory.

It must return exactly the verdicts of the allocating entry point voss_mr_verify_device, and a
seeded sample of them must equal the reference verifier's is_prime_u64 (compiled unmodified;
the oracle's restatement where that build is absent).  The
check runs on two calls in a row because every call shares the library's fixed scratch array
(the survivor work list and its counter): the second call must not see the first one's
leftovers.  This file is named to be collected last, so a run that stops at the first failure
has already run every other test; it also passes alone in a fresh process.
"""
import ctypes
import os

import numpy as np
import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

LIMIT = 1 << 22  # the entry point's per-call maximum


def _inputs(ctx, rng, count, lo):
    """Half known primes (sieved on the device), half random odd 64-bit values."""
    primes = ctx.primes_range(lo, lo + 40 * count)[: count // 2]
    odd = rng.integers(0, 2**63, size=count - primes.size, dtype=np.uint64) * 2 + 1
    n = np.concatenate([primes, odd])
    rng.shuffle(n)
    return n


def test_noalloc_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    import voss
    from voss import _native as N

    if voss.device_count() == 0 or not torch.cuda.is_available():
        pytest.fail("this GPU test ran without a CUDA device")
    lib = N.load()
    rng = np.random.default_rng(20261203)
    ctx = voss.Context(10**13)
    stream = torch.cuda.current_stream()
    # two calls in a row, the second at the maximum size
    for count, lo in ((1_000_003, 10**12), (LIMIT, 10**9)):
        n = _inputs(ctx, rng, count, lo)
        d_n = torch.from_numpy(n.view(np.int64)).to("cuda")
        want = torch.full((count,), 7, dtype=torch.uint8, device="cuda")
        got = torch.full((count,), 9, dtype=torch.uint8, device="cuda")
        ctx.mr_verify_device(d_n.data_ptr(), count, want.data_ptr(), stream.cuda_stream)
        rc = lib.voss_mr_verify_noalloc(ctypes.c_void_p(d_n.data_ptr()), count,
                                        ctypes.c_void_p(got.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, lib.voss_last_error()
        torch.cuda.synchronize()
        # integer verdicts: exact equality
        assert torch.equal(got, want)
        g = got.cpu().numpy()
        assert set(np.unique(g)) <= {0, 1}
        assert int(g.sum()) >= count // 2  # the known primes are all reported prime
        sample = rng.choice(count, 200_000, replace=False)
        ref = O.ref_mr_batch(n[sample]) if os.path.exists(O.REF_VERIFY_SO) else O.mr_batch(n[sample])
        np.testing.assert_array_equal(g[sample], ref)


def test_noalloc_rejects_oversize_and_null():
    torch = pytest.importorskip("torch")
    import voss
    from voss import _native as N

    if voss.device_count() == 0 or not torch.cuda.is_available():
        pytest.fail("this GPU test ran without a CUDA device")
    lib = N.load()
    buf = torch.zeros(16, dtype=torch.int64, device="cuda")
    rc = lib.voss_mr_verify_noalloc(ctypes.c_void_p(buf.data_ptr()), LIMIT + 1, ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == -1  # VOSS_ERR_ARG
    assert b"no-allocation limit" in lib.voss_last_error()
    assert lib.voss_mr_verify_noalloc(None, 5, ctypes.c_void_p(buf.data_ptr()), None) == -1
    assert lib.voss_mr_verify_noalloc(None, 0, None, None) == 0

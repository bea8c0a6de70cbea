"""Checkpoint / resume on the device: a run stopped by stop.txt and resumed equals one call."""
import os
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 10**10
SEG = 900_000_000  # 12 segments


def test_stop_and_resume_on_device(gpu_ctx):
    import voss
    whole = gpu_ctx.sieve_range(1, N + 1, compat=True, seg_num=SEG)
    with tempfile.TemporaryDirectory() as d:
        calls = []

        def seg(lo, hi):
            calls.append(lo)
            if len(calls) == 2:
                open(os.path.join(d, "stop.txt"), "w").close()
            return gpu_ctx.sieve_range(lo, hi, compat=True, seg_num=SEG)

        with pytest.raises(voss.VossError) as e:
            voss.run_checkpointed_fn(seg, N, SEG, True, 5, d)
        assert e.value.code == -7
        r, resumed = gpu_ctx.run_checkpointed(N, SEG, compat=True, ckpt_every=5, directory=d)
        assert resumed == 5  # saved after segment index 4 (schedule 0, 4, 9, 11)
        assert not os.path.exists(os.path.join(d, "checkpoint.bin"))
    for k in ("prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "large_total"):
        assert getattr(r, k) == getattr(whole, k), k
    for k in ("mod4", "modq", "modq_gap", "gap_hist"):
        np.testing.assert_array_equal(getattr(r, k), getattr(whole, k))
    assert sorted(r.large["position"].tolist()) == sorted(whole.large["position"].tolist())

"""Checkpoint / resume / stop file of the segment driver (voss_run_checkpointed_fn), on the
CPU: the segments come from the oracle, the driver logic (merging, checkpoint schedule and
format, stop file, resume) is the library's.  A resumed run must equal an uninterrupted one,
including the accumulators the reference's own checkpoint drops."""
import os
import struct
import tempfile

import numpy as np
import pytest

import oracle_lib as O
import voss

N = 30_000_000
SEG = 3_000_000  # 10 segments, a multiple of 30


def oracle_segment(lo, hi):
    return O.sieve_range(lo, hi, compat=True, seg_num=SEG)


def same(a, b):
    for k in ("lo", "hi", "prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "large_total"):
        assert getattr(a, k) == getattr(b, k), k
    for k in ("mod4", "modq", "modq_gap", "gap_hist"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    assert sorted(zip(a.large["position"].tolist(), a.large["gap"].tolist())) == \
        sorted(zip(b.large["position"].tolist(), b.large["gap"].tolist()))


def test_fresh_run_equals_single_range():
    with tempfile.TemporaryDirectory() as d:
        r, resumed = voss.run_checkpointed_fn(oracle_segment, N, SEG, True, 5, d)
        assert resumed == 0
        assert not os.path.exists(os.path.join(d, "checkpoint.bin"))  # removed on success
    same(r, O.sieve_range(1, N + 1, compat=True, seg_num=SEG))


def test_stop_file_then_resume_equals_fresh():
    with tempfile.TemporaryDirectory() as d:
        calls = []

        def seg(lo, hi):
            calls.append(lo)
            if len(calls) == 3:  # during segment index 2, ask the run to stop
                open(os.path.join(d, "stop.txt"), "w").close()
            return oracle_segment(lo, hi)

        with pytest.raises(voss.VossError) as e:
            voss.run_checkpointed_fn(seg, N, SEG, True, 2, d)
        assert e.value.code == -7
        assert os.path.exists(os.path.join(d, "checkpoint.bin"))
        assert not os.path.exists(os.path.join(d, "stop.txt"))  # consumed, as the reference does
        # the next save after the stop request is after segment index 3 (schedule: 0, 1, 3, 5, ...)
        assert len(calls) == 4
        r, resumed = voss.run_checkpointed_fn(oracle_segment, N, SEG, True, 2, d)
        assert resumed == 4
    same(r, O.sieve_range(1, N + 1, compat=True, seg_num=SEG))


def test_checkpoint_for_other_run_or_corrupt_is_ignored():
    with tempfile.TemporaryDirectory() as d:
        calls = []

        def seg(lo, hi):
            calls.append(lo)
            if len(calls) == 2:
                open(os.path.join(d, "stop.txt"), "w").close()
            return oracle_segment(lo, hi)

        with pytest.raises(voss.VossError):
            voss.run_checkpointed_fn(seg, N, SEG, True, 5, d)
        ck = os.path.join(d, "checkpoint.bin")
        assert os.path.exists(ck)
        # a different N must not resume from it
        r, resumed = voss.run_checkpointed_fn(oracle_segment, N - 30, SEG, True, 5, d)
        assert resumed == 0
        same(r, O.sieve_range(1, N - 30 + 1, compat=True, seg_num=SEG))
        # a damaged file is ignored too
        with open(ck, "wb") as f:
            f.write(b"VOSSCKP1" + struct.pack("<I", 99) + b"\0" * 64)
        r, resumed = voss.run_checkpointed_fn(oracle_segment, N, SEG, True, 5, d)
        assert resumed == 0
    same(r, O.sieve_range(1, N + 1, compat=True, seg_num=SEG))


def test_segment_errors_propagate():
    def bad(lo, hi):
        raise RuntimeError("simulated failure of a segment")

    with tempfile.TemporaryDirectory() as d:
        with pytest.raises(voss.VossError) as e:
            voss.run_checkpointed_fn(bad, N, SEG, True, 5, d)
        assert e.value.code == -9

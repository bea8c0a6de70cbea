"""Artifact parity with the reference program itself: src/voss_v7_live.cu compiled for sm_100a
(oracle/_ref/voss_v7_live_<N>, built by oracle/build_ref.py) runs in a temporary directory and
its CSVs and printed totals are compared with ours (voss_sieve_range in reference-compat mode +
voss_write_artifacts).  Every file must be byte-identical except large_gaps.csv, whose row
order the reference leaves to an unstable sort of equal merits; that one is compared as a set
of rows."""
import os
import re
import subprocess
import tempfile

import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

SEG = 30_000_000_000
EXACT = ["gap_histogram.csv", "hl_trend.csv", "modq_counts.csv", "modq_gap_hist.csv", "chebyshev.csv",
         "gap_sequence.csv"]


@pytest.mark.parametrize("n", [10**9, 10**10, 10**11, 10**12])
def test_artifacts_equal_reference_program(gpu_ctx, n):
    import voss
    exe = os.path.join(O.REF_BIN_DIR, f"voss_v7_live_{n}")
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built")
    with tempfile.TemporaryDirectory(prefix="vref_") as ref_dir, tempfile.TemporaryDirectory(prefix="vours_") as our_dir:
        r = subprocess.run([exe], cwd=ref_dir, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        res = gpu_ctx.sieve_range(1, n + 1, compat=True, seg_num=SEG, large_cap=50_000_000)
        voss.write_artifacts(res, our_dir)
        gap, p = gpu_ctx.gap_sequence(n, SEG, 5_000_000)
        voss.write_gap_sequence(gap, p, our_dir)
        m = re.search(r"Total primes:\s*(\d+)", r.stdout)
        assert m and int(m.group(1)) == res.prime_count
        for name in EXACT:
            a = open(os.path.join(ref_dir, name)).read()
            b = open(os.path.join(our_dir, name)).read()
            assert a == b, name
        ra = open(os.path.join(ref_dir, "large_gaps.csv")).read().splitlines()
        rb = open(os.path.join(our_dir, "large_gaps.csv")).read().splitlines()
        assert ra[0] == rb[0]
        assert sorted(ra[1:]) == sorted(rb[1:])
        # our order: merit descending (as the reference), ties by position
        merits = [float(x.split(",")[2]) for x in rb[1:]]
        assert merits == sorted(merits, reverse=True)

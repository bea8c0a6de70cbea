"""The drop-in drivers: voss/voss_master.py in place of the reference's src/voss_master.py, and
the voss_verify program in place of its bin/verify_cpp.  Both must leave the same files behind
as the reference, and print the same statistics block."""
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile

import pytest

import oracle_lib as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "voss-prime-gaps_v1_b200")
MASTER = os.path.join(PKG, "voss", "voss_master.py")
VERIFY = os.path.join(PKG, "voss", "_lib", "voss_verify")
GOLD = json.load(open(os.path.join(ROOT, "tests", "golden", "known_answers.json")))


def make_tree(d, n):
    """A reference-shaped tree: src/voss_master.py (ours, N rewritten the way run_voss.py
    rewrites it, run_voss.py:111-123), data/verification_db.json, results/."""
    os.makedirs(os.path.join(d, "src"))
    os.makedirs(os.path.join(d, "data"))
    src = open(MASTER).read()
    src = re.sub(r"(N_VALUE\s*=\s*)\d+", r"\g<1>" + str(n), src, count=1)
    open(os.path.join(d, "src", "voss_master.py"), "w").write(src)
    json.dump({"pi_of_10_pow_n": GOLD["pi_10n"]}, open(os.path.join(d, "data", "verification_db.json"), "w"))


def stats_block(text):
    a = text.index("=== Gap Statistics ===")
    b = text.index("[Check 3]")
    return text[a:b]


def test_voss_master_dropin_matches_reference_program():
    n = 10**9
    with tempfile.TemporaryDirectory() as d:
        make_tree(d, n)
        env = dict(os.environ, VOSS_PKG=PKG)
        r = subprocess.run([sys.executable, os.path.join(d, "src", "voss_master.py")], cwd=d, env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-3000:]
        assert "Total primes: 50847534" in r.stdout
        assert "\nPASS\n" in r.stdout
        assert r.stdout.count("-> PASS") == 3
        res = os.path.join(d, "results")
        for f in ("gap_histogram.csv", "hl_trend.csv", "modq_counts.csv", "modq_gap_hist.csv", "chebyshev.csv",
                  "large_gaps.csv"):
            assert os.path.exists(os.path.join(res, f)), f
        exe = os.path.join(O.REF_BIN_DIR, f"voss_v7_live_{n}")
        if os.path.exists(exe):
            with tempfile.TemporaryDirectory() as rd:
                rr = subprocess.run([exe], cwd=rd, capture_output=True, text=True, timeout=600)
                assert rr.returncode == 0
                assert stats_block(rr.stdout) == stats_block(r.stdout)
                for f in ("gap_histogram.csv", "hl_trend.csv", "modq_counts.csv", "modq_gap_hist.csv", "chebyshev.csv"):
                    assert open(os.path.join(rd, f)).read() == open(os.path.join(res, f)).read(), f


def test_voss_verify_dropin_matches_reference_verifier():
    import voss
    with tempfile.TemporaryDirectory() as d:
        res = os.path.join(d, "results")
        os.makedirs(res)
        with voss.Context(10**10 + 1) as ctx:
            r = ctx.sieve_range(1, 10**10 + 1, compat=True)
            voss.write_artifacts(r, res)
        rows = open(os.path.join(res, "large_gaps.csv")).read().splitlines()
        # two corrupted rows: a wrong gap and a composite end
        p, g, m = rows[1].split(",")
        rows.append(f"{p},{int(g) - 2},{m}")
        p, g, m = rows[2].split(",")
        rows.append(f"{int(p) + 2},{g},{m}")
        open(os.path.join(res, "large_gaps.csv"), "w").write("\n".join(rows) + "\n")
        ours = [VERIFY, "results/large_gaps.csv", "results/details_ours.csv", "results/cache_ours.csv"]
        r1 = subprocess.run(ours, cwd=d, capture_output=True, text=True, timeout=300)
        assert r1.returncode == 1, r1.stdout + r1.stderr   # two failures
        r2 = subprocess.run(ours, cwd=d, capture_output=True, text=True, timeout=300)
        assert r2.returncode == 1 and "Newly verify:  2" in r2.stdout  # the rest came from the cache
        ref = os.path.join(O.REF_BIN_DIR, "verify_cpp")
        if os.path.exists(ref):
            rr = subprocess.run([ref, "results/large_gaps.csv", "results/details_ref.csv", "results/cache_ref.csv"],
                                cwd=d, capture_output=True, text=True, timeout=300)
            assert rr.returncode == 1
            assert open(os.path.join(res, "details_ref.csv")).read() == open(os.path.join(res, "details_ours.csv")).read()
            assert open(os.path.join(res, "cache_ref.csv")).read() == open(os.path.join(res, "cache_ours.csv")).read()


def test_voss_master_sieves_once_whatever_the_large_gap_count(monkeypatch):
    """The drop-in's checkpointed run returns the large-gap list up to the reference's cap in
    one pass: no second sieve of [1, n] when the list outgrows a first guess.  With the cap
    set below the count, the list is cut at the cap as the reference cuts it at
    MAX_LARGE_GAPS (src/voss_v7_live.cu:292-294,809) and the count still reports all."""
    sys.path.insert(0, os.path.join(PKG, "voss"))
    import voss
    import voss_master as VM

    def no_second_sieve(*a, **k):
        raise AssertionError("voss_master sieved the range a second time")
    monkeypatch.setattr(voss.Context, "sieve_range", no_second_sieve)
    monkeypatch.setattr(voss.Context, "sieve_range_device", no_second_sieve)
    n = 10**9
    with tempfile.TemporaryDirectory() as d:
        full = VM.run(n=n, seg_num=30_000_000_000, results=d)["result"]
        assert full.prime_count == 50847534
        assert full.large.size == full.large_total == 296
    with tempfile.TemporaryDirectory() as d:
        cut = VM.run(n=n, seg_num=30_000_000_000, results=d, large_cap=100)["result"]
        assert cut.large_total == full.large_total and cut.large.size == 100
        rows = open(os.path.join(d, "large_gaps.csv")).read().strip().splitlines()
        assert len(rows) == 1 + 100
    ref = {(int(p), int(g)) for p, g in zip(full.large["position"], full.large["gap"])}
    assert {(int(p), int(g)) for p, g in zip(cut.large["position"], cut.large["gap"])} <= ref

#!/usr/bin/env python3
"""VOSS Master on the B200 library: a drop-in for the reference's src/voss_master.py.

The reference rewrites N/SEG_NUM/MAX_POS into src/voss_v7_live.cu, compiles it with nvcc, runs
the binary in RESULTS and parses its stdout (src/voss_master.py:88-179).  This driver keeps the
same module constants (run_voss.py:111-123 rewrites `N_VALUE = ...` and `SEG_NUM = ...` in this
file the same way), the same OEIS check and the same artifacts, but computes everything in
libvoss.so: the range segment by segment with checkpoint.bin / stop.txt in RESULTS
(voss_run_checkpointed, reference-compat statistics), the sampled gap sequence
(voss_gap_sequence), and the CSVs (voss_write_artifacts, voss_write_gap_sequence).  It prints
the reference program's report block, so the `Total primes:` line that the reference parses is
there too.

Placement: copy it over src/voss_master.py of the reference tree (ROOT is the parent of the
directory holding this file, as in the reference) and make the `voss` package importable
(PYTHONPATH or VOSS_PKG=<dir containing voss/>).
"""
import datetime
import json
import math
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, ".."))
DB_FILE = os.path.join(ROOT, "data", "verification_db.json")
RESULTS = os.environ.get("VOSS_RESULTS") or os.path.join(ROOT, "results")

# ============================================================
# settings — run_voss.py rewrites these two lines
# ============================================================
N_VALUE = 1000000000000    # 10^12
SEG_NUM = 30000000000      # 3x10^10 (the reference's segment length; used for its artifact rules)

MAX_LARGE_GAPS = 50_000_000  # src/voss_v7_live.cu:34
GAP_SEQ_SIZE = 5_000_000     # src/voss_v7_live.cu:35


def _import_voss():
    pkg = os.environ.get("VOSS_PKG")
    if pkg:
        sys.path.insert(0, pkg)
    try:
        import voss  # noqa: F401
    except ImportError:
        sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..")))
    import voss
    return voss


def ensure_db():
    """The OEIS table pi(10^n) (src/voss_master.py:31-54).  This build has no network: a
    missing database only disables the final check."""
    if os.path.exists(DB_FILE):
        db = json.load(open(DB_FILE))
        if len(db.get("pi_of_10_pow_n", {})) >= 10:
            print("DB OK: " + DB_FILE)
            return db
    print("No verification DB at " + DB_FILE + " (not downloaded by this driver)")
    return {"pi_of_10_pow_n": {}}


def detect_gpu():
    try:
        gpu = subprocess.run(["nvidia-smi", "--query-gpu=name,memory.total", "--format=csv,noheader"],
                             capture_output=True, text=True).stdout.strip().splitlines()[0]
        mem_gb = float(gpu.split(",")[1].strip().split()[0]) / 1024.0
    except (OSError, IndexError, ValueError):
        gpu, mem_gb = "unknown", 0.0
    return gpu, mem_gb, "sm_100a"


def run(n: int = None, seg_num: int = None, results: str = None, device: int = 0,
        large_cap: int = MAX_LARGE_GAPS) -> dict:
    """Sieve [1, n] in reference-compat mode, write the artifacts into `results`, print the
    reference's report; returns {"prime_count", "total_s", "result"}.

    The large-gap list keeps at most `large_cap` records, the reference's MAX_LARGE_GAPS
    (src/voss_v7_live.cu:34,292-294,809): the checkpointed run returns the whole list up to
    that cap in one pass (its host buffer is only touched where records are written), so
    [1, n] is sieved once whatever the number of large gaps."""
    voss = _import_voss()
    from voss.report import WRITTEN, report_lines
    n = N_VALUE if n is None else n
    seg_num = SEG_NUM if seg_num is None else seg_num
    results = RESULTS if results is None else results
    os.makedirs(results, exist_ok=True)
    t0 = time.perf_counter()
    num_seg = (n + seg_num - 1) // seg_num
    with voss.Context(n + 1, device=device) as ctx:
        # segment by segment with checkpoint.bin / stop.txt in the results directory, as the
        # reference program keeps them in its working directory (src/voss_v7_live.cu:407-421,599-621)
        try:
            res, resumed = ctx.run_checkpointed(n, seg_num, compat=True, ckpt_every=5, directory=results,
                                                large_cap=large_cap)
        except voss.VossError as e:
            if e.code == -7:  # stop file: checkpoint saved, clean exit (:603-620)
                print(f"\n>>> STOP-FILE detected — exiting cleanly <<<")
                return {"prime_count": None, "total_s": time.perf_counter() - t0, "result": None, "stopped": True}
            raise
        if resumed:
            print(f">>> RESUMING FROM SEGMENT {resumed} / {num_seg} <<<")
        else:
            print(">>> STARTING FRESH <<<")
        t_sieve = time.perf_counter() - t0
        gap, p = ctx.gap_sequence(n, seg_num, GAP_SEQ_SIZE)
    total_s = time.perf_counter() - t0
    voss.write_artifacts(res, results)
    voss.write_gap_sequence(gap, p, results)
    phases = [("Sieve", t_sieve), ("GapSeq", total_s - t_sieve)]
    for line in report_lines(res, total_s, phases, WRITTEN):
        print(line)
    print("\nDone.")
    return {"prime_count": res.prime_count, "total_s": total_s, "result": res}


def main():
    print("=" * 60)
    print("VOSS Master")
    print("=" * 60)
    print(f"ROOT  = {ROOT}")
    print()
    db = ensure_db()
    n_log10 = round(math.log10(N_VALUE))
    is_pow10 = abs(10**n_log10 - N_VALUE) / N_VALUE < 1e-9
    expected_pi = db["pi_of_10_pow_n"].get(str(n_log10)) if is_pow10 else None
    if expected_pi:
        print(f"pi(10^{n_log10}) from OEIS = {expected_pi:,}")
    print()
    gpu, mem_gb, arch = detect_gpu()
    print(f"GPU: {gpu}  arch={arch}")
    print(f"N={N_VALUE:,}  SEG_NUM={SEG_NUM:,}  NUM_SEG={math.ceil(N_VALUE / SEG_NUM)}")
    voss = _import_voss()
    print(f"Library: {voss.lib_path()} ({voss.version()})")
    print("=" * 60)
    print(f"Running in: {RESULTS}\n")
    out = run()
    actual = out["prime_count"]
    print("\n" + "=" * 60)
    print("=== AUTO-VERIFICATION vs OEIS A006880 ===")
    print("=" * 60)
    if actual and expected_pi:
        print(f"OEIS pi(10^{n_log10}) = {expected_pi:>25,}")
        print(f"VOSS pi(10^{n_log10}) = {actual:>25,}")
        d = actual - expected_pi
        print(f"Diff = {d:+,}")
        print("PASS" if d == 0 else f"FAIL ({d:,})")
    else:
        print("Verification skipped (not a power of 10, or parse failed).")
    print(f"[{datetime.datetime.now().isoformat(timespec='seconds')}]")


if __name__ == "__main__":
    main()

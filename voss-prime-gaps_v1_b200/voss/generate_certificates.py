#!/usr/bin/env python3
"""Gap certificates on the B200 library: a drop-in for the reference's
scripts/generate_certificates.py.

Reads results/large_gaps.csv and writes
  - results/certificates.csv: one row per gap, "p_before,p_after,gap,merit,sha256,verified"
    (scripts/generate_certificates.py:198-213), the digest being SHA-256 of
    "VOSS|p_before|p_after|gap|merit" with the merit printed to 6 decimals (:105-108);
  - results/cert_top20/cert_NN_merit<m>_p<p_after>.txt: text certificates of the 20 gaps of
    highest merit (:112-135, :216-225; ties keep file order).
The verdicts come from results/verification_details.csv when present (the verifier stage's
output, :161-170); gaps missing from it are proved on the GPU (voss_prove_gaps, the
reference's verify_gap).  All digests are computed in one GPU batch (voss_sha256_batch)
instead of one hashlib call per row.  The CSV is byte-identical to the reference script's;
the text certificates differ only in their "Generated:" time stamp.

Placement: copy it over scripts/generate_certificates.py of the reference tree (ROOT is the
parent of the directory holding this file) and make the `voss` package importable
(PYTHONPATH or VOSS_PKG=<dir containing voss/>).  VOSS_RESULTS overrides the results directory.
"""
import csv
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, ".."))
TOP_N = 20


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


def cert_message(p_before: int, p_after: int, gap: int, merit: float) -> bytes:
    """The hashed content of one certificate (scripts/generate_certificates.py:107)."""
    return f"VOSS|{p_before}|{p_after}|{gap}|{merit:.6f}".encode()


def cert_text(p_before: int, p_after: int, gap: int, merit: float, sha: str, stamp: str) -> str:
    """One text certificate, line for line the layout of scripts/generate_certificates.py:112-135."""
    bar, rule = "=" * 66, "-" * 66
    lines = [
        bar,
        "           VOSS NUMERICAL CERTIFICATE OF PRIME GAP",
        bar,
        f"Prime Before (p)        : {p_before:,}",
        f"Prime After  (p+g)      : {p_after:,}",
        f"Gap Size (g)            : {gap:,}",
        f"Merit (g / ln p)        : {merit:.6f}",
        f"ln(p)                   : {math.log(p_before):.6f}",
        f"Max Factor Limit (sqrtp+g) : {math.isqrt(p_after):,}",
        rule,
        "VERIFICATION METHOD:",
        "  1. p_before and p_after are proven prime via",
        "     Deterministic Miller-Rabin (bases 2,3,5,7,11,13,17,19,23,29,31,37).",
        f"  2. All {gap - 1} integers in (p, p+g) are proven composite",
        "     via Interval Sieve with base primes up to √(p+g).",
        rule,
        f"SHA-256: {sha}",
        f"Generated: {stamp}",
        bar,
    ]
    return "\n".join(lines) + "\n"


def run(results: str = None, device: int = 0) -> dict:
    voss = _import_voss()
    results = results or os.environ.get("VOSS_RESULTS") or os.path.join(ROOT, "results")
    src = os.path.join(results, "large_gaps.csv")
    out_csv = os.path.join(results, "certificates.csv")
    top_dir = os.path.join(results, "cert_top20")
    if not os.path.exists(src):
        print(f"ERROR: {src} not found")
        sys.exit(1)
    print(f"Reading: {src}")
    rows = []
    with open(src) as f:
        for r in csv.DictReader(f):
            rows.append((int(r["position"]), int(r["gap"]), float(r["merit"])))
    print(f"Gaps: {len(rows):,}")
    if not rows:
        print("Nothing to do")
        return {"rows": 0}
    t0 = time.time()
    details = os.path.join(results, "verification_details.csv")
    known = {}
    if os.path.exists(details):
        with open(details) as f:
            for r in csv.DictReader(f):
                known[(int(r["position"]), int(r["gap"]))] = r["verified"] == "1"
        print(f"  Loaded {len(known):,} verification results from {details}")
    import numpy as np
    with voss.Context(10**6, device=device) as ctx:
        todo = [i for i, (p, g, _) in enumerate(rows) if (p, g) not in known]
        verdict = {}
        if todo:
            print(f"  Proving {len(todo):,} gaps on the GPU")
            pa = np.array([rows[i][0] for i in todo], dtype=np.uint64)
            gp = np.array([rows[i][1] for i in todo], dtype=np.int32)
            ok = ctx.prove_gaps(pa, gp)
            verdict = {todo[k]: bool(ok[k]) for k in range(len(todo))}
        digests = ctx.sha256_batch([cert_message(p - g, p, g, m) for p, g, m in rows])
    shas = [d.tobytes().hex() for d in digests]
    verified = 0
    os.makedirs(results, exist_ok=True)
    with open(out_csv, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["p_before", "p_after", "gap", "merit", "sha256", "verified"])
        for i, (p, g, m) in enumerate(rows):
            ok = known[(p, g)] if (p, g) in known else verdict[i]
            verified += ok
            w.writerow([p - g, p, g, f"{m:.6f}", shas[i], "YES" if ok else "NO"])
    dt = time.time() - t0
    print(f"  Wrote {len(rows):,} certificates in {dt:.2f}s")
    print(f"  Verified: {verified:,}/{len(rows):,}")
    os.makedirs(top_dir, exist_ok=True)
    order = sorted(range(len(rows)), key=lambda i: -rows[i][2])[:TOP_N]  # stable: ties keep file order
    stamp = time.strftime("%Y-%m-%d %H:%M:%S")
    names = []
    for k, i in enumerate(order, 1):
        p, g, m = rows[i]
        name = f"cert_{k:02d}_merit{m:.2f}_p{p}.txt"
        with open(os.path.join(top_dir, name), "w", encoding="utf-8") as f:
            f.write(cert_text(p - g, p, g, m, shas[i], stamp))
        names.append(name)
        print(f"  [{k:2d}] {name}")
    print("\n" + "=" * 60)
    print("DIGITAL CERTIFICATES SUMMARY")
    print("=" * 60)
    print(f"  CSV  : {out_csv}")
    print(f"         {len(rows):,} certificates")
    print(f"  TXT  : {top_dir}/")
    print(f"         {TOP_N} top certificates by merit")
    print(f"  Time : {dt:.2f} s")
    print("=" * 60)
    return {"rows": len(rows), "verified": verified, "seconds": dt, "top": names}


if __name__ == "__main__":
    run()

"""The reference program's stdout report, printed from a RangeResult.

Line for line the end-of-run block of src/voss_v7_live.cu (:637-705 statistics and
self-checks, :711-733 and :750-783 "OK <file>" lines, :805-825 the large-gap list), with the
same printf formats, so that drivers that parse it (src/voss_master.py:170, `Total primes:`)
keep working.  The "Timing Breakdown" lists this engine's own phases instead of the reference's
sieve/extract/sort/mod-4/gaps kernels, which do not exist here.
"""
from __future__ import annotations

import math

import numpy as np


def gap_statistics(gap_hist: np.ndarray) -> dict:
    """Mean, standard deviation, skewness and excess kurtosis of the gap distribution,
    accumulated in the reference's order (voss_v7_live.cu:652-665)."""
    tgc = 0
    wsum = 0
    for g in range(1, gap_hist.size):
        c = int(gap_hist[g])
        tgc += c
        wsum += g * c
    mg = wsum / tgc if tgc else float("nan")
    vs = ss = ks = 0.0
    for g in range(1, gap_hist.size):
        c = int(gap_hist[g])
        if c == 0:
            continue
        d = float(g) - mg
        vs += float(c) * d * d
        ss += float(c) * d * d * d
        ks += float(c) * d * d * d * d
    var = vs / float(tgc) if tgc else float("nan")
    sd = math.sqrt(var) if tgc else float("nan")
    sk = ss / float(tgc) / (var * sd) if tgc and var > 0 else float("nan")
    ku = ks / float(tgc) / (var * var) - 3.0 if tgc and var > 0 else float("nan")
    return {"tgc": tgc, "wsum": wsum, "mean": mg, "sd": sd, "skew": sk, "kurt": ku}


def report_lines(res, total_s: float, phases: list[tuple[str, float]], written: list[str]) -> list[str]:
    g = res.gap_hist
    st = gap_statistics(g)
    out = []
    out.append("=" * 61)
    out.append(f"TOTAL TIME: {total_s:.2f} s ({total_s / 60.0:.2f} min)")
    out.append(f"Total primes: {res.prime_count}")
    out.append("=" * 61)
    out.append("")
    out.append("=== Timing Breakdown ===")
    accounted = 0.0
    for name, sec in phases:
        accounted += sec
        pct = 100.0 * sec / total_s if total_s > 0 else 0.0
        out.append(f"{name + ':':<11}{sec:10.2f} s ({pct:6.2f}%)")
    other = total_s - accounted
    out.append(f"{'Other:':<11}{other:10.2f} s ({(100.0 * other / total_s if total_s > 0 else 0.0):6.2f}%)")
    out.append("")
    out.append("=== Gap Statistics ===")
    out.append(f"Total gaps:  {st['tgc']}")
    out.append(f"Mean gap:    {st['mean']:.4f}")
    out.append(f"Std dev:     {st['sd']:.4f}")
    out.append(f"Skewness:    {st['skew']:.4f}")
    out.append(f"Kurtosis:    {st['kurt']:.4f}")
    out.append("")
    out.append("=== Gap Counts ===")
    for k, pad in ((1, "  "), (2, "  "), (4, "  "), (6, "  "), (12, " "), (30, " ")):
        out.append(f"Gap {k}:{pad}{int(g[k])}")
    out.append("")
    p41, p43 = int(res.mod4[0]), int(res.mod4[1])
    out.append("=== Chebyshev Bias ===")
    out.append(f"pi(x;4,1) = {p41}")
    out.append(f"pi(x;4,3) = {p43}")
    out.append(f"Diff      = {p43 - p41}")
    out.append("")
    p6p2 = float(g[6]) / float(g[2]) if g[2] else float("nan")
    out.append("=== Gap Repulsion ===")
    out.append(f"P(6)/P(2) = {p6p2:.6f}")
    out.append("")
    tp = res.prime_count
    out.append("=== Self-Consistency Checks ===")
    out.append("[Check 1] sum(N(g)) = pi(N) - 1")
    out.append(f"  sum(N(g))  = {st['tgc']}")
    out.append(f"  pi(N) - 1  = {tp - 1}")
    out.append(f"  -> {'PASS' if st['tgc'] == tp - 1 else 'FAIL'}")
    out.append("[Check 2] sum(g*N(g)) = p_last - 2")
    out.append(f"  sum(g*N(g)) = {st['wsum']}")
    out.append(f"  p_last - 2  = {res.last_prime - 2}")
    out.append(f"  -> {'PASS' if st['wsum'] == res.last_prime - 2 else 'FAIL'}")
    out.append("[Check 3] pi(4,1) + pi(4,3) + 1 = pi(N)")
    out.append(f"  pi41+pi43+1 = {p41 + p43 + 1}")
    out.append(f"  pi(N)       = {tp}")
    out.append(f"  -> {'PASS' if p41 + p43 + 1 == tp else 'FAIL'}")
    out.append("")
    for w in written:
        out.append(w)
    lg = res.large
    out.append("")
    out.append("=== Large Gaps (>= 500) ===")
    out.append(f"Count: {res.large_total}")
    if lg.size:
        order = sorted(range(lg.size), key=lambda i: (-float(lg["merit"][i]), int(lg["position"][i])))
        out.append(f"OK large_gaps.csv ({lg.size} entries)")
        for i in order[:10]:
            out.append(f"  gap={int(lg['gap'][i]):4d} merit={float(lg['merit'][i]):6.2f} at p={int(lg['position'][i])}")
    else:
        out.append("OK large_gaps.csv (0 entries)")
    return out


WRITTEN = ["OK gap_histogram.csv", "OK hl_trend.csv (hybrid)", "OK modq_counts.csv", "OK modq_gap_hist.csv",
           "OK chebyshev.csv", "OK gap_sequence.csv"]

#!/usr/bin/env python3
"""Regenerate the golden fixtures in this directory from the reference tree.

Reads (never copies wholesale) the reference's committed known answers:
  results/hist_snapshots/hist_<N>.csv   full gap histograms at N = 1e3, 1e11, 1e12, 1e13, 1e14
  data/verification_db.json             pi(10^n) (OEIS A006880)
  README.md Chebyshev table             pi(x;4,1), pi(x;4,3) for x = 10^9 .. 10^14
  results/modq_counts.csv               mod-6 / mod-30 prime counts at N = 1e14
  results/modq_gap_hist.csv             per-residue gap histogram (gaps < 100) at N = 1e14
  results/chebyshev.csv, hl_trend.csv   the N = 1e14 artifacts
and writes them as compact fixtures that the tests read on machines without the reference.

usage: python tests/golden/make_golden.py [--ref REFERENCE_CHECKOUT]  (default: $VOSS_REF)
"""
import argparse
import csv
import json
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
SUP = str.maketrans("⁰¹²³⁴⁵⁶⁷⁸⁹", "0123456789")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("VOSS_REF"), required=not os.environ.get("VOSS_REF"))
    a = ap.parse_args()
    ref = a.ref
    out = {}
    # pi(10^n)
    db = json.load(open(os.path.join(ref, "data", "verification_db.json")))
    out["pi_10n"] = {k: int(v) for k, v in db["pi_of_10_pow_n"].items() if int(k) <= 19}
    # histograms
    hists = {}
    snap = os.path.join(ref, "results", "hist_snapshots")
    for fn in sorted(os.listdir(snap)):
        m = re.match(r"hist_(\d+)\.csv$", fn)
        if not m:
            continue
        rows = list(csv.DictReader(open(os.path.join(snap, fn))))
        hists[m.group(1)] = {r["gap"]: int(r["count"]) for r in rows}
    out["gap_hist"] = hists
    # Chebyshev table from the README
    cheb = {}
    for line in open(os.path.join(ref, "README.md"), encoding="utf-8"):
        m = re.match(r"\|\s*10([⁰¹²³⁴⁵⁶⁷⁸⁹]+)\s*\|\s*([\d,]+)\s*\|\s*([\d,]+)\s*\|\s*\*\*\+?([\d,]+)\*\*", line)
        if m:
            e = int(m.group(1).translate(SUP))
            cheb[str(10**e)] = [int(m.group(2).replace(",", "")), int(m.group(3).replace(",", ""))]
    out["chebyshev"] = cheb
    # N = 1e14 artifacts
    res = os.path.join(ref, "results")
    out["modq_counts_1e14"] = [[int(r["q"]), int(r["a"]), int(r["count"])]
                               for r in csv.DictReader(open(os.path.join(res, "modq_counts.csv")))]
    out["modq_gap_hist_1e14"] = [[int(r["q"]), int(r["residue"]), int(r["gap"]), int(r["count"])]
                                 for r in csv.DictReader(open(os.path.join(res, "modq_gap_hist.csv")))]
    out["hl_trend_fixed"] = [[int(r["N"]), r["P6_over_P2"]]
                             for r in csv.DictReader(open(os.path.join(res, "hl_trend.csv")))][:5]
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "known_answers.json"))


if __name__ == "__main__":
    main()

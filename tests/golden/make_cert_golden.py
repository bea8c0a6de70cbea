#!/usr/bin/env python3
"""Regenerate the certificate fixtures from the reference's own certificate generator.

Runs scripts/generate_certificates.py of the reference tree (imported from there; it needs
numba) on a small large-gap list and stores what it writes:
  cert_large_gaps_1e9.csv    the input: the large gaps below 1e9 (reference-compat statistics of
                             the CPU oracle, written by voss_write_artifacts in the reference's
                             large_gaps.csv format) plus a few altered rows that fail their proof
  cert_certificates_1e9.csv  the reference's certificates.csv for that input (no
                             verification_details.csv: it proves every row itself)
  cert_top20_1e9.json        its top-20 text certificates, file name -> content, each without
                             its "Generated:" time-stamp line

usage: python tests/golden/make_cert_golden.py [--ref REFERENCE_CHECKOUT]  (default: $VOSS_REF)
"""
import argparse
import importlib.util
import json
import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("VOSS_REF"), required=not os.environ.get("VOSS_REF"))
    a = ap.parse_args()
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, os.path.join(ROOT, "voss-prime-gaps_v1_b200"))
    import oracle_lib as O
    import voss
    spec = importlib.util.spec_from_file_location("ref_generate_certificates",
                                                  os.path.join(a.ref, "scripts", "generate_certificates.py"))
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    with tempfile.TemporaryDirectory() as d:
        res = os.path.join(d, "results")
        os.makedirs(res)
        r = O.sieve_range(1, 10**9 + 1, compat=True, seg_num=30_000_000_000)
        voss.write_artifacts(r, res)
        lines = open(os.path.join(res, "large_gaps.csv")).read().splitlines()
        rows = [ln.split(",") for ln in lines[1:]]
        extra = []
        for pos, gap, merit in rows[:3]:
            extra.append(f"{int(pos) + 2},{gap},{merit}")          # p_after not prime
            extra.append(f"{pos},{int(gap) - 2},{merit}")          # p_before not prime
            extra.append(f"{pos},{int(gap) + int(rows[-1][1])},{merit}")  # longer: interior holds a prime or ends fail
        text = "\n".join(lines + extra) + "\n"
        src = os.path.join(res, "large_gaps.csv")
        open(src, "w").write(text)
        for name in os.listdir(res):
            if name != "large_gaps.csv":
                os.remove(os.path.join(res, name))
        ref.ROOT = d
        ref.INPUT = src
        ref.CERT_CSV = os.path.join(res, "certificates.csv")
        ref.TOP20_DIR = os.path.join(res, "cert_top20")
        ref.main()
        shutil.copyfile(src, os.path.join(HERE, "cert_large_gaps_1e9.csv"))
        shutil.copyfile(ref.CERT_CSV, os.path.join(HERE, "cert_certificates_1e9.csv"))
        top = {}
        for name in sorted(os.listdir(ref.TOP20_DIR)):
            body = open(os.path.join(ref.TOP20_DIR, name), encoding="utf-8").read().splitlines(keepends=True)
            top[name] = "".join(ln for ln in body if not ln.startswith("Generated: "))
        with open(os.path.join(HERE, "cert_top20_1e9.json"), "w", encoding="utf-8") as f:
            json.dump(top, f, indent=1, ensure_ascii=False)
    print("wrote cert_large_gaps_1e9.csv, cert_certificates_1e9.csv, cert_top20_1e9.json")


if __name__ == "__main__":
    main()

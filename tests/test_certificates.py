"""Certificate formats on the CPU: the hashed message and the text certificate of the drop-in
voss/generate_certificates.py against the fixtures written by the reference's own
scripts/generate_certificates.py (tests/golden/make_cert_golden.py); digests by hashlib here,
the GPU digests are checked in test_gpu_cert.py."""
import csv
import hashlib
import json
import os

from voss import generate_certificates as G

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rows():
    with open(os.path.join(GOLD, "cert_large_gaps_1e9.csv")) as f:
        return [(int(r["position"]), int(r["gap"]), float(r["merit"])) for r in csv.DictReader(f)]


def test_message_digests_match_reference_output():
    rows = _rows()
    with open(os.path.join(GOLD, "cert_certificates_1e9.csv"), newline="") as f:
        want = list(csv.DictReader(f))
    assert len(want) == len(rows) == 305
    for (p, g, m), w in zip(rows, want):
        assert (int(w["p_before"]), int(w["p_after"]), int(w["gap"]), w["merit"]) == (p - g, p, g, f"{m:.6f}")
        assert hashlib.sha256(G.cert_message(p - g, p, g, m)).hexdigest() == w["sha256"]


def test_text_certificates_match_reference_output():
    rows = _rows()
    top = json.load(open(os.path.join(GOLD, "cert_top20_1e9.json"), encoding="utf-8"))
    order = sorted(range(len(rows)), key=lambda i: -rows[i][2])[:20]
    names = []
    for k, i in enumerate(order, 1):
        p, g, m = rows[i]
        name = f"cert_{k:02d}_merit{m:.2f}_p{p}.txt"
        names.append(name)
        sha = hashlib.sha256(G.cert_message(p - g, p, g, m)).hexdigest()
        text = G.cert_text(p - g, p, g, m, sha, "2000-01-01 00:00:00")
        body = "".join(ln for ln in text.splitlines(keepends=True) if not ln.startswith("Generated: "))
        assert body == top[name], name
    assert sorted(names) == sorted(top)

"""GPU certificate hashing: voss_sha256_batch against hashlib on messages of every length
around the SHA-256 block boundaries, and the drop-in voss/generate_certificates.py against the
files the reference's own scripts/generate_certificates.py wrote for the same input
(tests/golden/make_cert_golden.py): certificates.csv byte for byte, the top-20 text
certificates except their time-stamp line."""
import hashlib
import json
import os
import shutil
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_sha256_batch_matches_hashlib(gpu_ctx):
    rng = np.random.default_rng(11)
    lens = list(range(0, 200)) + [255, 256, 257, 447, 448, 1000, 4096] + list(rng.integers(0, 300, 5000))
    msgs = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes() for n in lens]
    got = gpu_ctx.sha256_batch(msgs)
    want = np.array([np.frombuffer(hashlib.sha256(m).digest(), dtype=np.uint8) for m in msgs])
    np.testing.assert_array_equal(got, want)
    assert gpu_ctx.sha256_batch([]).shape == (0, 32)


def test_dropin_certificates_equal_reference_files():
    from voss import generate_certificates as G
    with tempfile.TemporaryDirectory() as d:
        shutil.copyfile(os.path.join(GOLD, "cert_large_gaps_1e9.csv"), os.path.join(d, "large_gaps.csv"))
        out = G.run(results=d)
        assert out["rows"] == 305 and out["verified"] == 296
        got = open(os.path.join(d, "certificates.csv"), "rb").read()
        assert got == open(os.path.join(GOLD, "cert_certificates_1e9.csv"), "rb").read()
        top = json.load(open(os.path.join(GOLD, "cert_top20_1e9.json"), encoding="utf-8"))
        names = sorted(os.listdir(os.path.join(d, "cert_top20")))
        assert names == sorted(top)
        for name in names:
            body = open(os.path.join(d, "cert_top20", name), encoding="utf-8").read().splitlines(keepends=True)
            assert "".join(ln for ln in body if not ln.startswith("Generated: ")) == top[name], name

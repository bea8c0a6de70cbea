"""The bounds-checked build (libvoss_checked.so: every shared-memory index of the sieve kernel is
checked, and a bad one is recorded in the error word instead of being accessed) runs the
sieve's main workloads in a separate process (among them a range of 33,000 tiles, so that
every CTA runs hundreds of tiles with its double-buffered tile headers): no call may report a bounds error, and every
result must equal the product library's."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "voss-prime-gaps_v1_b200", "voss", "_lib")

CHILD = r'''
import hashlib, json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np, voss
h = hashlib.sha1()
with voss.Context(10**18 + 2 * 10**9) as ctx:
    r = ctx.sieve_range(1, 10**9 + 1, compat=True)
    for k in ("gap_hist", "mod4", "modq", "modq_gap"):
        h.update(np.ascontiguousarray(getattr(r, k)).tobytes())
    h.update(np.sort(r.large["position"]).tobytes())
    # a long range: hundreds of tiles per CTA
    r2 = ctx.sieve_range(10**11, 3 * 10**11)
    for k in ("gap_hist", "mod4", "modq", "modq_gap"):
        h.update(np.ascontiguousarray(getattr(r2, k)).tobytes())
    h.update(np.sort(r2.large["position"]).tobytes())
    rng = np.random.default_rng(3)
    lo = (np.floor(10 ** rng.uniform(3, 18, 300))).astype(np.uint64)
    hi = lo + np.floor(10 ** rng.uniform(1, 7, 300)).astype(np.uint64)
    iv = ctx.sieve_intervals(lo, hi)
    h.update(iv.tobytes())
    g = ctx.gaps_at_least(10**12, 10**12 + 10**9, 300)
    h.update(np.sort(g["position"]).tobytes())
    p = ctx.primes_range(10**15, 10**15 + 10**6)
    h.update(p.tobytes())
print(json.dumps({"hash": h.hexdigest(), "pi": r.prime_count}))
'''


def _run(lib):
    env = dict(os.environ, VOSS_LIB=os.path.join(LIBDIR, lib))
    out = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "voss-prime-gaps_v1_b200")],
                         env=env, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_checked_build_reports_nothing_and_matches():
    if not os.path.exists(os.path.join(LIBDIR, "libvoss_checked.so")):
        pytest.skip("libvoss_checked.so not built")
    a = _run("libvoss.so")
    b = _run("libvoss_checked.so")
    assert a == b and a["pi"] == 50847534

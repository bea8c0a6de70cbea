"""Autotuner for the interval work queue.

For a batch of intervals it picks the sieve tuning (tile shape = block_threads x chunk_words,
the small/medium prime split coop_div, the multiples-walk threshold mult_factor) by timing a
fixed candidate set on a sample of the batch's interval-size classes, with the kernel time
the library measures (voss_last_kernel_ms).  Results are cached per (device, size-class
signature) in a JSON file so that later batches of the same shape reuse them.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

# candidate tunings: tile bytes from 200 KB (1 CTA/SM) down to 36 KB (several CTAs/SM), with the
# small/medium split (coop_div) and the pre-pass threshold (mult_factor) near their measured optima
CANDIDATES = [
    dict(block_threads=1024, chunk_words=49, coop_div=80, mult_factor=8),
    dict(block_threads=1024, chunk_words=49, coop_div=64, mult_factor=8),
    dict(block_threads=1024, chunk_words=49, coop_div=64, mult_factor=16),
    dict(block_threads=1024, chunk_words=25, coop_div=64, mult_factor=8),
    dict(block_threads=512, chunk_words=45, coop_div=64, mult_factor=8),
    dict(block_threads=512, chunk_words=21, coop_div=32, mult_factor=8),
    dict(block_threads=512, chunk_words=9, coop_div=16, mult_factor=4),
]

CLASS_EDGES = (10**5, 10**6, 10**7)  # interval lengths: tiny / small / medium / large


def size_classes(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    return np.searchsorted(np.array(CLASS_EDGES, dtype=np.float64), (hi - lo).astype(np.float64), side="right")


def signature(lo: np.ndarray, hi: np.ndarray) -> str:
    c = size_classes(lo, hi)
    frac = np.bincount(c, minlength=len(CLASS_EDGES) + 1) / max(1, c.size)
    mag = int(np.round(np.log10(max(float(hi.max()), 10.0))))
    return "mag%d:" % mag + ",".join("%.1f" % f for f in frac)


def _cache_path() -> str:
    return os.environ.get("VOSS_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "voss_tune.json"))


def tune_intervals(ctx, lo, hi, sample: int = 512, reps: int = 2, seed: int = 1, use_cache: bool = True,
                   candidates=None) -> dict:
    """Choose and apply the best candidate tuning for batches shaped like (lo, hi).

    Returns {"tuning": ..., "timings_ms": {...}, "signature": ..., "cached": bool}."""
    lo = np.ascontiguousarray(lo, dtype=np.uint64)
    hi = np.ascontiguousarray(hi, dtype=np.uint64)
    sig = signature(lo, hi)
    dev = "%s/%d" % (ctx.info()["sm_count"], ctx.device)
    key = dev + "|" + sig
    path = _cache_path()
    cache = {}
    if use_cache and os.path.exists(path):
        try:
            cache = json.load(open(path))
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache:
        ctx.set_tuning(**cache[key]["tuning"])
        return dict(cache[key], cached=True)
    rng = np.random.default_rng(seed)
    idx = rng.choice(lo.size, size=min(sample, lo.size), replace=False)
    slo, shi = lo[idx], hi[idx]
    timings = {}
    best, best_ms = None, float("inf")
    for cand in candidates or CANDIDATES:
        try:
            ctx.set_tuning(**cand)
        except Exception:
            continue
        ctx.sieve_intervals(slo, shi)  # warm-up
        ms = []
        for _ in range(reps):
            ctx.sieve_intervals(slo, shi)
            ms.append(ctx.last_kernel_ms()[1])
        t = float(np.median(ms))
        name = "%dx%d/c%d/m%d" % (cand["block_threads"], cand["chunk_words"], cand["coop_div"], cand["mult_factor"])
        timings[name] = t
        if t < best_ms:
            best, best_ms = cand, t
    ctx.set_tuning(**best)
    res = {"tuning": best, "timings_ms": timings, "signature": sig, "when": time.time()}
    if use_cache:
        cache[key] = res
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            json.dump(cache, open(path, "w"), indent=1)
        except OSError:
            pass
    return dict(res, cached=False)

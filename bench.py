#!/usr/bin/env python3
"""Benchmark: wheel-30 sieve + fused gap statistics of [1, 10^12] on B200.

Workload (one "step"): sieve every integer of [1, N] (N = 10^12 by default) and compute the
reference's statistics in reference-compat mode: pi(N), the gap histogram, mod-4 / mod-q
counts, the per-residue gap histogram, the large-gap list and the maximal gap.  Metric:
range/s = integers sieved per second (higher is better).

  value      device time of the sieve+stitch+reduce kernels per step (CUDA events on the
             launching stream, L2 flushed between steps outside the timed events), max over
             ranks; inputs (base-prime table) resident in HBM.
  e2e        the same step through the public C ABI call voss_sieve_range with host result
             buffers (device->host copy of the statistics and large-gap list inside the
             timed region), wall clock, max over ranks; for N > 1 it includes the NCCL
             all-gather of the per-rank statistics and their merge on rank 0.
  roofline   dominant kernel sieve_tiles_kernel against the device's measured shared-memory
             read-modify-write bandwidth (the sieve never touches HBM).
  cpu_baseline  the oracle's OpenMP interval sieve (a restatement of the reference's
             verify_cpp marking loop) on a bounded sample of the same range, rank 0, N = 1.
  ref_cuda   the reference's voss_v7_live.cu rebuilt for sm_100a (oracle/_ref), its printed
             TOTAL TIME at the same N (rank 0, N = 1), when the binary is present.

  roofline_split  the tile kernel's time split into its sieve and extraction phases (phase
             shares from the phase-timing build, run in a child process), each against the
             same shared-memory peak.

At 1 GPU the line also carries the other halves of the metric, each a complete sub-line with
its own value, e2e, roofline, clocks and baseline (same --steps / --warmup):
  intervals  4096 seeded intervals (a log-uniform [1e10, 1e16], L log-uniform [1e4, 1e8]) in
             one batched persistent launch versus one plain launch per interval;
  mr         10^8 Miller-Rabin candidates (5e7 primes below 1e12 + 5e7 random odd u64) and the
             interior proofs of all gaps >= 200 below 1e12, beside the reference verifier;
  serve      seeded Poisson request streams at 1e2, 1e3, 1e4 req/s through the
             continuous-batching server (p50/p99) versus plain launches, and the capacity of
             both with every request offered at once (capacity_ratio_vs_plain).
`--workload intervals|mr|serve` prints one of them alone; `--sub ""` leaves them out.

Multi-GPU (torchrun): weak scaling; rank r sieves [r*N + 1, (r+1)*N], the statistics are
all-gathered over NCCL and merged (voss_stats_merge) into those of [1, world*N].

`--impl reference` times the reference's CPU path for this workload (see cpu_baseline) and
prints the same metric.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "voss-prime-gaps_v1_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

SEG_NUM = 30_000_000_000
METRIC = "range/s sieved to 1e12 (sieve + fused gap/mod-q statistics)"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=10**12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU sample duration")
    ap.add_argument("--workload", default="range", choices=["range", "intervals", "mr", "serve"],
                    help="range: sieve+stats of [1, n] (headline); intervals: 4096 seeded intervals")
    ap.add_argument("--intervals", type=int, default=4096)
    ap.add_argument("--mr-half", type=int, default=50_000_000, help="known primes (= random odds) in the MR batch")
    ap.add_argument("--no-gap-proofs", action="store_true")
    ap.add_argument("--rates", default="100,1000,10000", help="serving: Poisson arrival rates (req/s)")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="serving: length of each arrival stream")
    ap.add_argument("--plain-seconds", type=float, default=20.0, help="serving: cap on the plain-launch replay")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="intervals: skip the one-launch-per-interval comparison")
    ap.add_argument("--capacity-requests", type=int, default=20000,
                    help="serving: requests offered at once for the capacity comparison")
    ap.add_argument("--sub", default="intervals,mr,serve",
                    help="range workload at 1 GPU: the other workloads to run after it and attach to its line "
                         "(comma list of intervals, mr, serve; empty for none)")
    ap.add_argument("--no-extract-split", action="store_true")
    ap.add_argument("--phase-probe", action="store_true", help=argparse.SUPPRESS)
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return json.load(open(p))
    except (OSError, ValueError):
        return {}


def profile_traffic_per_unit() -> tuple[float | None, str | None]:
    """DRAM bytes per sieved integer of sieve_tiles_kernel from the committed ncu summary."""
    rel = os.path.join("profiles", "sieve_tiles_kernel_1e11.md")
    try:
        txt = open(os.path.join(ROOT, rel)).read()
    except OSError:
        return None, None
    m = re.search(r"dram_bytes_per_integer:\s*([0-9.eE+-]+)", txt)
    return (float(m.group(1)), rel + " (10^11 capture, scaled by integers)") if m else (None, None)


_COPRIME30 = [sum(1 for r in range(1, x + 1) if r % 2 and r % 3 and r % 5) for x in range(30)]


def sieve_work(n: int) -> int:
    """H(n): bit-clears of the wheel-30 sieve of [1, n] — for every prime 7 <= p <= isqrt(n),
    the multiples of p in [p^2, n] that are coprime to 30 (the reference's per-prime start
    rule, voss_v7_live.cu:449-478).  Numpy, so the roofline needs nothing from the oracle."""
    import numpy as np
    s = math.isqrt(n)
    if s < 7:
        return 0
    flags = np.ones(s + 1, dtype=bool)
    flags[:2] = False
    for q in range(2, math.isqrt(s) + 1):
        if flags[q]:
            flags[q * q::q] = False
    p = np.nonzero(flags)[0].astype(np.int64)
    p = p[p >= 7]
    table = np.asarray(_COPRIME30, dtype=np.int64)

    def upto(x):
        return 8 * (x // 30) + table[x % 30]
    return int((upto(n // p) - upto(p - 1)).sum())


def primes_upto(s: int):
    """Primes 7 <= p <= s as float64 (numpy sieve of Eratosthenes)."""
    import numpy as np
    flags = np.ones(s + 1, dtype=bool)
    flags[:2] = False
    for q in range(2, math.isqrt(s) + 1):
        if flags[q]:
            flags[q * q::q] = False
    p = np.nonzero(flags)[0]
    return p[p >= 7].astype(np.float64)


def interval_work(lo, hi, p_large: int, mr_route: int = 50) -> dict:
    """Algorithmic work terms of a batch of intervals [lo_i, hi_i).

    offsets: one first-hit computation per (interval, base prime 7 <= p <= isqrt(hi_i - 1)).
    Bit-clears: for each such prime, the multiples of p in [max(lo_i, p^2), hi_i) coprime to 30,
    taken as their expected count 8 (hi_i - max(lo_i, p^2)) / (30 p); split into the primes
    7..31 (applied as word masks, no clears), 37 <= p < p_large (cleared in shared memory by the
    tile kernel) and p >= p_large (the large-prime pre-pass).  Expected rather than exact counts:
    exact ones would take one division per (interval, prime), ~10^10 on the host here."""
    import numpy as np
    P = primes_upto(math.isqrt(int(hi.max()) - 1))
    inv = np.concatenate([[0.0], np.cumsum(1.0 / P)])
    cuts = [7.0, 37.0, float(p_large), math.inf]  # presieve | tile | pre-pass
    offsets = 0
    hits = [0.0, 0.0, 0.0]
    for a, b in zip(lo.tolist(), hi.tolist()):
        if b <= a:
            continue
        s_hi = math.isqrt(b - 1)
        s_lo = math.isqrt(a)  # p <= s_lo: p^2 <= lo, multiples from lo
        n_hi = int(np.searchsorted(P, s_hi, side="right"))
        n_lo = min(int(np.searchsorted(P, s_lo, side="right")), n_hi)
        offsets += n_hi
        big = P[n_lo:n_hi]  # lo < p^2 < hi: multiples from p^2
        for c in range(3):
            i0 = int(np.searchsorted(P, cuts[c], side="left"))
            i1 = int(np.searchsorted(P, cuts[c + 1], side="left")) if cuts[c + 1] != math.inf else P.size
            j1 = min(i1, n_lo)
            if j1 > i0:
                hits[c] += (b - a) * (inv[j1] - inv[i0])
            sel = big[(big >= cuts[c]) & (big < cuts[c + 1])]
            if sel.size:
                hits[c] += float(((b - sel * sel) / sel).sum())
    # (prime, interval) pairs of the large-prime pre-pass: primes p_large <= p <= isqrt(hi - 1) of
    # every interval the library sieves (those with more base primes than mr_route times their
    # length go to Miller-Rabin instead, the rule of voss_sieve_intervals)
    n_large_lt = int(np.searchsorted(P, float(p_large), side="left"))
    pairs = routed = 0
    for a, b in zip(lo.tolist(), hi.tolist()):
        a7 = max(a, 7)
        if b <= a7:
            continue
        np_hi = int(np.searchsorted(P, math.isqrt(b - 1), side="right"))
        if mr_route != 0xFFFFFFFF and b - a7 < (1 << 31) and np_hi // mr_route > b - a7:
            routed += 1
            continue
        pairs += max(0, np_hi - n_large_lt)
    k = 8.0 / 30.0
    return {"first_hit_offsets": int(offsets), "presieve_primes_hits": k * hits[0],
            "tile_hits": k * hits[1], "prepass_hits": k * hits[2], "p_large": int(p_large),
            "prepass_pairs": int(pairs), "mr_routed_intervals": int(routed),
            "note": "hits are expected counts, 8(hi - max(lo, p^2))/(30p) per (interval, prime)"}


_MR_BASES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def mr_mulmods(sample) -> tuple[int, int]:
    """Montgomery products the Miller-Rabin kernels' algorithm needs for these candidates,
    (moduli below 2^63, moduli above): per candidate that trial division by 2..37 leaves open,
    for each base in order up to the first that fails, or up to as many bases as n's size needs
    (6, 7, 9 or 12): one squaring per bit of the odd part d, one product per set bit of d (none
    for base 2, whose products are doublings), and the squarings of the r - 1 follow-up steps
    up to the first -1.  The lanes' padding in the warp-uniform loops is overhead, not counted."""
    small = full = 0
    for n in map(int, sample):
        if n < 2 or n % 2 == 0 or any(n == b or n % b == 0 for b in _MR_BASES[1:]):
            continue
        d = n - 1
        r = (d & -d).bit_length() - 1
        d >>= r
        bits, ones = d.bit_length(), bin(d).count("1")
        need = 6 if n < 3474749660383 else 7 if n < 341550071728321 else 9 if n < 3825123056546413051 else 12
        cnt = 0
        for a in _MR_BASES[:need]:
            cnt += bits + (0 if a == 2 else ones)
            x = pow(a, d, n)
            ok = x == 1 or x == n - 1
            j = 0
            while not ok and j < r - 1:
                x = x * x % n
                j += 1
                cnt += 1
                ok = x == n - 1
            if not ok:
                break
        if n < 1 << 63:
            small += cnt
        else:
            full += cnt
    return small, full


# ---------------------------------------------------------------------------------------
def sample_slices(n: int, span: int, k: int = 8) -> list[tuple[int, int]]:
    """A stratified sample of [1, n]: k slices of span/k integers, slice j centred in the j-th of
    k equal parts, so the sample's rate is that of the whole range (the CPU sieve slows as the
    base primes grow towards isqrt(n))."""
    w = max(1, span // k)
    out = []
    for j in range(k):
        c = 1 + (2 * j + 1) * n // (2 * k)
        lo = max(1, min(c - w // 2, n + 1 - w))
        out.append((lo, lo + w))
    return out


def time_slices(slices, threads: int) -> float:
    import oracle_lib as O
    t0 = time.perf_counter()
    for lo, hi in slices:
        O.sieve_range(lo, hi, compat=True, seg_num=SEG_NUM, threads=threads)
    return time.perf_counter() - t0


def describe_slices(slices) -> str:
    w = slices[0][1] - slices[0][0]
    return (f"{len(slices)} slices of {w:.3e} integers centred in the {len(slices)} equal parts of the range "
            f"(first [{slices[0][0]}, {slices[0][1]}), last [{slices[-1][0]}, {slices[-1][1]}))")


def cpu_baseline(n: int, seconds: float) -> dict:
    """Oracle OpenMP interval sieve (port of verify_cpp's marking loop) on a stratified sample of
    [1, n] sized to about `seconds` of CPU work."""
    import oracle_lib as O
    threads = O.oracle().oracle_max_threads()
    probe = sample_slices(n, 2 * 10**8)
    rate = sum(h - l for l, h in probe) / max(time_slices(probe, threads), 1e-6)
    sl = sample_slices(n, int(min(n, max(2 * 10**8, rate * seconds))))
    dt = time_slices(sl, threads)
    total = sum(h - l for l, h in sl)
    return {"value": total / dt, "unit": "range/s", "cores": threads, "kind": "port",
            "sample": f"oracle interval sieve + statistics, {describe_slices(sl)}, {total:.3e} integers, "
                      f"{dt:.1f} s, OpenMP {threads} threads"}


def ref_cuda_baseline(n: int) -> dict | None:
    exe = os.path.join(ROOT, "oracle", "_ref", f"voss_v7_live_{n}")
    if not os.path.exists(exe):
        return None
    with tempfile.TemporaryDirectory(prefix="voss_ref_run_") as d:
        t0 = time.perf_counter()
        r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=900)
        wall = time.perf_counter() - t0
    m = re.search(r"TOTAL TIME:\s*([0-9.]+)\s*s", r.stdout)
    pi = re.search(r"Total primes:\s*(\d+)", r.stdout)
    if r.returncode != 0 or not m:
        return {"unavailable": f"reference binary rc={r.returncode}"}
    t = float(m.group(1))
    return {"value": n / t, "unit": "range/s", "total_time_s": t, "wall_s": round(wall, 2),
            "pi": int(pi.group(1)) if pi else None,
            "what": "reference src/voss_v7_live.cu rebuilt with nvcc -O3 -arch=sm_100a, its TOTAL TIME"}


# ---------------------------------------------------------------------------------------
def range_workload(n: int) -> str:
    return f"wheel-30 sieve + reference statistics of [1, {n}] per GPU (REF_COMPAT, SEG_NUM={SEG_NUM})"


def run_reference_arm(a) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle_lib as O
    threads = O.oracle().oracle_max_threads()
    # one step = a bounded stratified sample (about 4 s of CPU work) of [1, n]
    probe = sample_slices(a.n, 10**8)
    rate = sum(h - l for l, h in probe) / max(time_slices(probe, threads), 1e-6)
    sl = sample_slices(a.n, int(min(a.n, max(10**8, rate * 4.0))))
    span = sum(h - l for l, h in sl)
    for _ in range(a.warmup):
        time_slices(sl, threads)
    times = [time_slices(sl, threads) for _ in range(a.steps)]
    ms = 1e3 * statistics.mean(times)
    value = span / (ms * 1e-3)
    sample = f"oracle interval sieve + statistics per step: {describe_slices(sl)} ({span:.3e} integers)"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "range/s", "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (the integer range itself)",
        "config": {"workload": range_workload(a.n), "n_per_gpu": a.n, "range": [1, a.n],
                   "parallelism": f"host CPU, {threads} threads (rank 0 only)"},
        "cpu_baseline": {"value": value, "unit": "range/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "range/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def interval_batch(k: int, seed: int = 20261203):
    """4096 intervals [a, a+L): a log-uniform in [1e10, 1e16] rounded down to a multiple of
    30, L log-uniform in [1e4, 1e8] (numpy PCG64, fixed seed)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    a = (np.floor(10 ** rng.uniform(10, 16, k) / 30) * 30).astype(np.uint64)
    ln = np.floor(10 ** rng.uniform(4, 8, k)).astype(np.uint64)
    return a, a + ln


def run_intervals(a) -> dict:
    """Batched uneven intervals: one persistent launch over the (interval, tile) work queue
    versus one plain launch per interval; results must agree bit for bit."""
    import numpy as np
    import voss
    from voss.autotune import tune_intervals
    import torch
    lo, hi = interval_batch(a.intervals)
    ctx = voss.Context(int(hi.max()) + 1)
    tune = None if a.no_tune else tune_intervals(ctx, lo, hi, use_cache=False)
    for _ in range(a.warmup):
        ctx.sieve_intervals(lo, hi)
    # the base-prime table (69 MB) fits in L2: flush it between timed steps
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda:0")
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    dev_ms, wall, phases = [], [], []
    for _ in range(a.steps):
        flush.add_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        batched = ctx.sieve_intervals(lo, hi)
        wall.append(time.perf_counter() - t0)
        dev_ms.append(ctx.last_kernel_ms()[1])
        phases.append(ctx.last_phase_ms())
    clk = clocks.stop()
    # one plain launch per interval
    plain_wall = 0.0
    plain_dev = 0.0
    plain = batched.copy() if a.no_plain else np.zeros_like(batched)
    for i in range(0 if a.no_plain else lo.size):
        t0 = time.perf_counter()
        plain[i] = ctx.sieve_intervals(lo[i:i + 1], hi[i:i + 1])[0]
        plain_wall += time.perf_counter() - t0
        plain_dev += ctx.last_kernel_ms()[1]
    same = all(np.array_equal(batched[f], plain[f]) for f in
               ("prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "gap_overflow", "gap_hist"))
    total_int = float((hi - lo).sum())
    bw = statistics.mean(wall)
    bd = statistics.mean(dev_ms) * 1e-3
    pre_ms, tile_ms, tail_ms = (statistics.mean(ph[k] for ph in phases) for k in range(3))
    t = ctx.tuning()
    tile_bytes = 4 * t["block_threads"] * t["chunk_words"]
    work = interval_work(lo, hi, t["mult_factor"] * tile_bytes, t["mr_route"])
    smem_peak = ctx.probe_smem_rmw()
    # tile kernel: 8 B per shared-memory bit-clear + one read of the intervals' bitmap words
    alg_bytes = 8.0 * work["tile_hits"] + total_int / 30.0
    achieved = alg_bytes / (tile_ms * 1e-3) / 1e9
    out = {
        "metric": "mixed-interval queries/s (4096 seeded intervals, batched persistent launch)",
        "value": lo.size / bd, "unit": "intervals/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": bd * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic: a log-uniform [1e10,1e16] (multiple of 30), L log-uniform [1e4,1e8], PCG64 seed 20261203",
        "config": {"workload": "batched intervals", "intervals": int(lo.size), "integers": total_int,
                   "tuning": ctx.tuning(), "autotune": tune,
                   "l2": "flushed (256 MiB write) between timed steps"},
        "integers_per_s": total_int / bd,
        "e2e": {"value": lo.size / bw, "unit": "intervals/s", "h2d_bytes_per_step": 48 * int(lo.size),
                "d2h_bytes_per_step": batched.itemsize * int(lo.size) + 32},
        "phases_ms": {"copies_memsets_prepass": pre_ms, "tile_kernel": tile_ms, "stitch_reduce_finalize": tail_ms},
        "work_terms": work,
        "prepass_clears_per_s": work["prepass_hits"] / (pre_ms * 1e-3) if pre_ms > 0 else None,
        "prepass": {
            "bound": "int", "pairs": work["prepass_pairs"],
            "pairs_per_s": work["prepass_pairs"] / (pre_ms * 1e-3) if pre_ms > 0 else None,
            "ms": pre_ms, "clears": work["prepass_hits"],
            "issue_frac_ncu": 0.722, "alu_frac_ncu": 0.587,
            "source": "issue and ALU-pipe fractions of peak (active cycles) of scatter_large_kernel from the "
                      "committed capture profiles/scatter_large_kernel_intervals.md; one 64-bit reduction per "
                      "(prime, interval) pair, ms includes the batch's copies and bitmap memset"},
        "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                     "frac": achieved / smem_peak, "traffic": None, "kernel": "sieve_tiles_kernel",
                     "kernel_ms": tile_ms, "algorithmic_bytes": alg_bytes,
                     "peak_source": "voss_probe_smem_rmw (this GPU, this run)",
                     "traffic_note": "DRAM traffic of this launch: profiles/launches_intervals_4096.md"},
        "clocks": clk,
        "gpu_launches": a.steps * phases[-1][3],
    }
    if not a.no_plain:
        out["plain_launch_per_interval"] = {"value": lo.size / plain_dev * 1e3, "unit": "intervals/s (device)",
                                            "e2e_value": lo.size / plain_wall, "total_device_ms": plain_dev,
                                            "total_wall_s": plain_wall}
        out["speedup_vs_plain"] = {"device": plain_dev / (bd * 1e3), "e2e": plain_wall / bw}
        out["bit_exact_vs_plain"] = bool(same)
    del ctx
    return out


def mr_candidates(ctx, half: int, seed: int = 20261203):
    """half consecutive primes just below 1e12 (the sieve's own output) + half uniformly random
    odd 64-bit values (PCG64, fixed seed), interleaved by a seeded permutation."""
    import numpy as np
    span = int(half * 28.5) + 10**6
    p = ctx.primes_range(10**12 - span, 10**12)[-half:]
    rng = np.random.default_rng(seed)
    r = rng.integers(0, 2**63, size=half, dtype=np.uint64) * 2 + 1
    n = np.concatenate([p, r])
    perm = rng.permutation(n.size)
    return n[perm], perm < p.size


def run_mr(a) -> dict:
    """Batched verification: 1e8 candidates through deterministic Miller-Rabin (12 bases), and
    the interior-composite proof of every gap >= 200 below 1e12."""
    import numpy as np
    import torch
    import voss
    import oracle_lib as O
    ctx = voss.Context(10**12 + 1)
    half = a.mr_half
    n, known = mr_candidates(ctx, half)
    d_n = torch.from_numpy(n.view(np.int64)).cuda()
    d_out = torch.empty(n.size, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()  # a real stream handle: 0 would select the context's own stream
    torch.cuda.synchronize()
    for _ in range(a.warmup):
        ctx.mr_verify_device(d_n.data_ptr(), n.size, d_out.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    for e0, e1 in ev:
        e0.record(stream)
        ctx.mr_verify_device(d_n.data_ptr(), n.size, d_out.data_ptr(), stream.cuda_stream)
        e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    # roofline: Montgomery products the algorithm needs (counted on a seeded sample of the
    # batch, scaled) against this GPU's measured product rate, per modulus class
    msample = n[: min(n.size, 100_000)]
    m_small, m_full = mr_mulmods(msample)
    scale = n.size / msample.size
    m_small, m_full = m_small * scale, m_full * scale
    peak_full, peak_small = ctx.probe_mulmod()
    t_ideal = m_small / peak_small + m_full / peak_full
    t_meas = ms * 1e-3
    got = d_out.cpu().numpy()
    # e2e through the host-buffer entry point
    t0 = time.perf_counter()
    for _ in range(a.steps):
        host = ctx.mr_verify(n)
    e2e = (time.perf_counter() - t0) / a.steps
    same_host = bool(np.array_equal(host, got))
    # CPU baseline: the reference verifier's is_prime_u64 (compiled unmodified) on a sample
    import os as _os
    sample = n[: 2_000_000]
    use_ref = _os.path.exists(O.REF_VERIFY_SO)
    thr = O.ref_verify().ref_max_threads() if use_ref else O.oracle().oracle_max_threads()
    t0 = time.perf_counter()
    ref = O.ref_mr_batch(sample) if use_ref else O.mr_batch(sample)
    cpu_s = time.perf_counter() - t0
    match = bool(np.array_equal(ref, got[: sample.size]))
    # gap proofs: every gap >= 200 below 1e12
    proofs = None
    if not a.no_gap_proofs:
        gaps = ctx.gaps_at_least(1, 10**12 + 1, 200)
        p_after = gaps["position"].astype(np.uint64)
        g = gaps["gap"].astype(np.int32)
        ctx.prove_gaps(p_after[:1000], g[:1000])
        t0 = time.perf_counter()
        ok = ctx.prove_gaps(p_after, g)
        prove_s = time.perf_counter() - t0
        ps = np.arange(0, p_after.size, max(1, p_after.size // 20000))[:20000]
        t0 = time.perf_counter()
        ref_ok = O.ref_prove_gaps(p_after[ps], g[ps]) if use_ref else O.prove_gaps(p_after[ps], g[ps])
        cpu_prove_s = time.perf_counter() - t0
        proofs = {"gaps_ge_200_below_1e12": int(p_after.size), "all_verified": bool(ok.all()),
                  "gpu_s": prove_s, "gpu_gaps_per_s": p_after.size / prove_s,
                  "cpu_reference_gaps_per_s": ps.size / cpu_prove_s, "cpu_cores": thr,
                  "cpu_sample": int(ps.size), "cpu_matches_gpu": bool(np.array_equal(ref_ok, ok[ps]))}
    out = {
        "metric": "Miller-Rabin candidates/s (1e8 candidates: 5e7 primes below 1e12 + 5e7 random odd u64)",
        "value": n.size / (ms * 1e-3), "unit": "candidates/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: sieved primes + PCG64 seed 20261203 odd values",
        "config": {"workload": "batched Miller-Rabin, bases 2..37, 64-bit Montgomery", "candidates": int(n.size),
                   "known_primes": int(known.sum())},
        "e2e": {"value": n.size / e2e, "unit": "candidates/s", "h2d_bytes_per_step": 8 * int(n.size),
                "d2h_bytes_per_step": int(n.size), "api": "voss_mr_verify (host buffers)"},
        "primes_found": int(got.sum()), "known_primes_all_prime": bool(got[known].all()),
        "host_equals_device": same_host,
        "cpu_baseline": {"value": sample.size / cpu_s, "unit": "candidates/s", "cores": thr,
                         "kind": "reference" if use_ref else "port",
                         "sample": f"first {sample.size} candidates through verify_cpp.cpp is_prime_u64",
                         "matches_gpu": match},
        "gap_proofs": proofs,
        "roofline": {"bound": "int", "achieved": (m_small + m_full) / t_meas / 1e9,
                     "peak": (m_small + m_full) / t_ideal / 1e9, "unit": "G Montgomery products/s",
                     "frac": t_ideal / t_meas, "traffic": None,
                     "kernel": "mr_sieve_kernel + mr_finish_kernel (one call)", "kernel_ms": ms,
                     "products_per_candidate": (m_small + m_full) / n.size,
                     "products_small_modulus": m_small, "products_full_modulus": m_full,
                     "peak_small_per_s": peak_small, "peak_full_per_s": peak_full,
                     "peak_source": "voss_probe_mulmod: independent Montgomery squaring chains on this GPU in "
                                    "this run (moduli < 2^63 and >= 2^63); peak = the products' time-weighted rate",
                     "count_sample": int(msample.size),
                     "traffic_note": "8 B read + 1 B written per candidate; mr_finish_kernel DRAM figures in "
                                     "profiles/mr_finish_kernel_2e6.md"},
        "clocks": clk,
        "gpu_launches": 2 * a.steps,
    }
    del ctx
    return out


def run_serve(a) -> dict:
    """Serving: seeded Poisson streams of mixed requests (70% interval sieve + gap statistics,
    start log-uniform [1e9, 1e18], length log-uniform [1e3, 1e9]; 30% Miller-Rabin batches of
    10^U(3,6) odd u64) through the continuous-batching server, versus the same stream served with
    one plain launch per request.  Then the capacity of both: the same kind of requests all
    offered at once (arrival times zero), served by the server and one at a time by plain
    launches; capacity_ratio_vs_plain = served req/s / plain req/s."""
    import numpy as np
    import voss
    from voss.serve import Server, request_stream, serve_plain, serve_stream
    ctx = voss.Context(10**18 + 10**9 + 1)
    # warm-up: kernels, tables, slots
    with Server(ctx) as srv:
        serve_stream(srv, request_stream(1e4, 200, seed=1))
    rows = []
    for rate in [float(x) for x in a.rates.split(",")]:
        count = int(min(30000, max(50, rate * a.serve_seconds)))
        stream = request_stream(rate, count, seed=20261203)
        clocks = ClockSampler(0)
        clocks.start()
        with Server(ctx) as srv:
            lat, wall, _, err = serve_stream(srv, stream)
            st = srv.stats()
        clk = clocks.stop()
        done = lat[~np.isnan(lat)]
        # the same stream served one request at a time with plain launches, in arrival order,
        # until the time cap (latency from arrival, so it includes queueing behind earlier ones)
        pl, plain_wall = serve_plain(ctx, stream, time_cap=a.plain_seconds)
        plain_n = len(pl)
        rows.append({
            "rate_req_s": rate, "requests": count, "errors": len(err),
            "p50_ms": float(np.percentile(done, 50) * 1e3), "p99_ms": float(np.percentile(done, 99) * 1e3),
            "mean_ms": float(done.mean() * 1e3), "throughput_req_s": count / wall,
            "batches": st["batches"], "mean_batch_requests": st["mean_batch_requests"],
            "max_inflight_batches": st["max_inflight_batches"], "clocks": clk,
            "plain": {"requests_served": plain_n, "p50_ms": float(np.percentile(pl, 50) * 1e3),
                      "p99_ms": float(np.percentile(pl, 99) * 1e3), "throughput_req_s": plain_n / plain_wall,
                      "note": "one request at a time in arrival order (time-capped replay of the same stream); "
                              "latency from arrival includes the wait behind earlier requests"},
        })
        del stream
    # capacity: every request offered at time zero (request_stream draws the arrival gaps first,
    # so these payloads are those of the 1e4 req/s stream of the same length and seed)
    cap_n = a.capacity_requests
    burst = request_stream(1e12, cap_n, seed=20261203)
    clocks = ClockSampler(0)
    clocks.start()
    runs = []
    for _ in range(3):  # the best of three runs (all reported): host scheduling and the copies vary
        with Server(ctx) as srv:
            lat, wall, _, err = serve_stream(srv, burst)
            st = srv.stats()
        runs.append((wall, lat, err, st))
    clk = clocks.stop()
    wall, lat, err, st = min(runs, key=lambda r: r[0])
    done = lat[~np.isnan(lat)]
    pl, plain_wall = serve_plain(ctx, burst, time_cap=a.plain_seconds)
    served_rps, plain_rps = cap_n / wall, len(pl) / plain_wall
    capacity = {"requests": cap_n, "errors": len(err), "served_req_s": served_rps, "served_wall_s": wall,
                "served_runs_wall_s": [r[0] for r in runs],
                "served_p50_ms": float(np.percentile(done, 50) * 1e3),
                "served_p99_ms": float(np.percentile(done, 99) * 1e3),
                "batches": st["batches"], "mean_batch_requests": st["mean_batch_requests"],
                "plain_req_s": plain_rps, "plain_requests_served": len(pl), "plain_wall_s": plain_wall,
                "clocks": clk,
                "note": "all requests offered at once (the payloads of the 1e4 req/s stream of this length); "
                        "served = continuous batching over 4 slots, the best of three runs; plain = one launch "
                        "per request in order (time-capped); both include the host copies of the requests"}
    top = rows[-1]
    out = {
        "metric": "serving: completed requests/s with p50/p99 latency (continuous batching)",
        "value": top["throughput_req_s"], "unit": "req/s", "n_gpus": 1, "steps": len(rows), "warmup": 1,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic: seeded Poisson arrivals (PCG64 seed 20261203)",
        "config": {"workload": "mixed interval + Miller-Rabin requests", "slots": 4, "base_primes_to": "1e9"},
        "rates": rows,
        "capacity": capacity,
        "capacity_ratio_vs_plain": served_rps / plain_rps,
    }
    del ctx
    return out


def extract_split(n: int) -> dict | None:
    """Share of the tile kernel's time in each phase, from the phase-timing build
    (libvoss_timing.so: a block barrier and a clock64 stamp at every phase boundary), run in a
    child process so that it does not replace the product library in this one."""
    lib = os.path.join(ROOT, "voss-prime-gaps_v1_b200", "voss", "_lib", "libvoss_timing.so")
    if not os.path.exists(lib):
        return None
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--phase-probe", "--n", str(n)],
                       capture_output=True, text=True, timeout=600)
    try:
        return json.loads(r.stdout.strip().splitlines()[-1])
    except (ValueError, IndexError):
        return {"unavailable": f"phase probe rc={r.returncode}: {r.stderr.strip()[-200:]}"}


PHASES = ("claim_flush", "header", "fill", "small_primes", "medium_primes", "large_primes", "restore",
          "extract_scan", "extract_walk", "extract_reduce")


def run_phase_probe(n: int) -> None:
    """Child process of extract_split: one REF_COMPAT sieve of [1, n] through the timing build."""
    import ctypes
    import voss
    from voss import _native as N
    lib = os.path.join(ROOT, "voss-prime-gaps_v1_b200", "voss", "_lib", "libvoss_timing.so")
    ctx = voss.Context(n + 1, lib_path=lib)
    L = ctx.lib
    L.voss_debug_phase_cycles.argtypes = [ctypes.POINTER(ctypes.c_ulonglong), ctypes.c_int, ctypes.c_int]
    ctx.sieve_range(1, 10**9 + 1, compat=True, seg_num=SEG_NUM)  # warm-up
    buf = (ctypes.c_ulonglong * 10)()
    N.check(L.voss_debug_phase_cycles(buf, 10, 1))
    ctx.sieve_range(1, n + 1, compat=True, seg_num=SEG_NUM)
    N.check(L.voss_debug_phase_cycles(buf, 10, 1))
    cyc = [int(x) for x in buf]
    tot = float(sum(cyc)) or 1.0
    print(json.dumps({"cycles": dict(zip(PHASES, cyc)), "share": {k: c / tot for k, c in zip(PHASES, cyc)},
                      "timing_build_ms": ctx.last_kernel_ms()[1]}), flush=True)


def main():
    a = parse()
    if a.phase_probe:
        run_phase_probe(a.n)
        return
    if a.impl == "reference":
        run_reference_arm(a)
        return
    if a.workload in ("intervals", "mr", "serve"):
        fn = {"intervals": run_intervals, "mr": run_mr, "serve": run_serve}[a.workload]
        print(json.dumps(fn(a)), flush=True)
        return
    import numpy as np
    import torch
    import voss

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    def barrier():
        if dist is not None:
            dist.barrier(device_ids=[local])
        torch.cuda.synchronize()

    n = a.n
    lo, hi = rank * n + 1, (rank + 1) * n + 1
    ctx = voss.Context(world * n + 1, device=local)
    stream = torch.cuda.Stream(device=local)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=f"cuda:{local}")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]

    # warm-up (W untimed steps)
    for _ in range(a.warmup):
        with torch.cuda.stream(stream):
            ctx.sieve_range_device(lo, hi, compat=True, seg_num=SEG_NUM, stream=stream.cuda_stream)
        stream.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    # ---- value: device-resident steps ----------------------------------------------------
    barrier()
    sieve_ms = []
    for k in range(a.steps):
        with torch.cuda.stream(stream):
            flush.add_(1)  # write > L2 between steps, outside the timed events
            ev[k][0].record(stream)
            ctx.sieve_range_device(lo, hi, compat=True, seg_num=SEG_NUM, stream=stream.cuda_stream)
            ev[k][1].record(stream)
        stream.synchronize()
        ph = ctx.last_phase_ms()
        sieve_ms.append(ph[1])  # the tile kernel alone
        step_kernels = ph[3]
    barrier()
    step_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    kernel_ms = statistics.mean(sieve_ms)
    # ---- e2e: through the public C ABI with host buffers ---------------------------------
    barrier()
    t0 = time.perf_counter()
    last = None
    for k in range(a.steps):
        r = ctx.sieve_range(lo, hi, compat=True, seg_num=SEG_NUM)
        if world > 1:
            blob = torch.frombuffer(bytearray(bytes(r.raw)), dtype=torch.uint8).to(f"cuda:{local}")
            gathered = [torch.empty_like(blob) for _ in range(world)]
            dist.all_gather(gathered, blob)
            if rank == 0:
                parts = []
                for gt in gathered:
                    st = voss._native.RangeStats.from_buffer_copy(gt.cpu().numpy().tobytes())
                    parts.append(voss.range_result(st))
                merged = voss.merge_stats(parts)
                last = merged
        else:
            last = r
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / a.steps
    barrier()
    clk = clocks.stop()

    t_step = torch.tensor([step_ms, e2e_s, kernel_ms], dtype=torch.float64, device=f"cuda:{local}")
    if dist is not None:
        dist.all_reduce(t_step, op=dist.ReduceOp.MAX)
    step_ms, e2e_s, kernel_ms = t_step.tolist()

    if rank != 0:
        del ctx
        if dist is not None:
            dist.destroy_process_group()
        return

    total_range = world * n
    value = total_range / (step_ms * 1e-3)
    # algorithmic bytes of the dominant kernel: 8 B per bit-clear (32-bit RMW) + one read of
    # the bitmap (N/30 B) by the extraction, for this rank's range
    h = sieve_work(hi - 1) - (sieve_work(lo - 1) if lo > 1 else 0)
    alg_bytes = 8.0 * h + (hi - lo) / 30.0
    smem_peak = ctx.probe_smem_rmw()
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    tpu, tsrc = profile_traffic_per_unit()
    peaks = measured_peaks()
    r = last
    d2h = 32 + 32 + 2800 * 8 + 16 * int(min(r.large_total, 1 << 22)) if r is not None else 0
    out = {
        "metric": METRIC, "value": value, "unit": "range/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (the integer range itself)",
        "config": {"workload": range_workload(n), "n_per_gpu": n,
                   "range": [1, total_range], "l2": "flushed (256 MiB write) between timed steps",
                   "tuning": ctx.tuning(), "parallelism": f"range-sharded x{world}"},
        "e2e": {"value": total_range / e2e_s, "unit": "range/s", "h2d_bytes_per_step": 48,
                "d2h_bytes_per_step": d2h, "api": "voss_sieve_range (host buffers)"},
        "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                     "frac": achieved / smem_peak, "traffic": (tpu * (hi - lo)) if tpu else None,
                     "kernel": "sieve_tiles_kernel", "kernel_ms": kernel_ms,
                     "algorithmic_bytes": alg_bytes, "bit_clears": h,
                     "peak_source": "voss_probe_smem_rmw: bank-conflict-free shared-memory atomicAnd on "
                                    "this GPU in this run (8 B per 32-bit RMW); MEASURED_PEAKS.json has no "
                                    "shared-memory entry",
                     "hbm_peak_measured_gbs": peaks.get("hbm_gbs"),
                     "traffic_source": tsrc},
        "clocks": clk,
        "gpu_launches": step_kernels * a.steps,
        "result": {"pi": r.prime_count if r else None, "max_gap": r.max_gap if r else None,
                   "large_gaps": r.large_total if r else None},
    }
    if world == 1:
        if not a.no_extract_split:
            sp = extract_split(n)
            if sp and "share" in sp:
                sh = sp["share"]
                ext = sh["extract_scan"] + sh["extract_walk"] + sh["extract_reduce"]
                sie = sh["fill"] + sh["small_primes"] + sh["medium_primes"] + sh["large_primes"] + sh["restore"]
                # extraction: two 32-bit reads of every bitmap word (N/30 B each: the residue-class
                # count by word and the in-order walk) + one 32-bit shared-memory RMW per prime (its
                # gap bin, 8 B) + 64 RMWs per 1001 words (the class counters)
                ext_bytes = 2.0 * (hi - lo) / 30.0 + 8.0 * r.prime_count + 8.0 * 64.0 * (hi - lo) / (120.0 * 1001.0)
                ext_ms, sie_ms = ext * kernel_ms, sie * kernel_ms
                out["roofline_split"] = {
                    "source": "phase shares of the tile kernel from the phase-timing build (libvoss_timing.so, "
                              "clock64 stamps summed over CTAs) applied to this run's kernel_ms",
                    "phase_share": sh,
                    "sieve": {"ms": sie_ms, "algorithmic_bytes": 8.0 * h,
                              "achieved": 8.0 * h / (sie_ms * 1e-3) / 1e9, "peak": smem_peak, "unit": "GB/s",
                              "frac": 8.0 * h / (sie_ms * 1e-3) / 1e9 / smem_peak,
                              "phases": "fill, small/medium/large primes, restore"},
                    "extract": {"ms": ext_ms, "algorithmic_bytes": ext_bytes,
                                "achieved": ext_bytes / (ext_ms * 1e-3) / 1e9, "peak": smem_peak, "unit": "GB/s",
                                "frac": ext_bytes / (ext_ms * 1e-3) / 1e9 / smem_peak,
                                "bytes_note": "2 N/30 B of bitmap reads + 8 B (one 32-bit RMW) per prime + 64 RMWs per 1001 words",
                                "phases": "last-prime scan, in-order walk with counters, tile reduce"},
                }
            elif sp:
                out["roofline_split"] = sp
        if not a.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(n, a.cpu_seconds)
        if not a.no_ref_cuda:
            rc = ref_cuda_baseline(n)
            if rc is not None:
                out["ref_cuda"] = rc
        del ctx
        subs = {"intervals": run_intervals, "mr": run_mr, "serve": run_serve}
        for name in [x for x in a.sub.split(",") if x]:
            out[name] = subs[name](a)
        print(json.dumps(out), flush=True)
        return
    print(json.dumps(out), flush=True)
    del ctx
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

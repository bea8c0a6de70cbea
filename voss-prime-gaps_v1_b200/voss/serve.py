"""Python face of the request server (voss_server_* in include/voss.h) and a seeded
Poisson load generator for it."""
from __future__ import annotations

import ctypes
import threading
import time
from ctypes import byref, c_double, c_uint64, c_void_p

import numpy as np

from . import _native as N
from .api import INTERVAL_DTYPE, Context


class Server:
    """voss_server over a Context: thread-safe submit/wait/result; close() drains and stops."""

    def __init__(self, ctx: Context, slots: int = 4, max_batch_requests: int = 1024, max_batch_tiles: int = 1 << 16,
                 max_batch_candidates: int = 1 << 22, fail_every_n_batches: int = 0):
        self.ctx = ctx
        self.lib = N.load()
        cfg = N.ServerConfig(slots=slots, max_batch_requests=max_batch_requests, max_batch_tiles=max_batch_tiles,
                             fail_every_n_batches=fail_every_n_batches, max_batch_candidates=max_batch_candidates)
        h = c_void_p()
        N.check(self.lib.voss_server_create(ctx.handle, byref(cfg), byref(h)))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self.lib.voss_server_destroy(self._h)
            self._h = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit_interval(self, lo: int, hi: int) -> int:
        t = c_uint64()
        N.check(self.lib.voss_server_submit_interval(self._h, lo, hi, byref(t)))
        return t.value

    def submit_mr(self, n) -> tuple[int, int]:
        n = np.ascontiguousarray(n, dtype=np.uint64)
        t = c_uint64()
        N.check(self.lib.voss_server_submit_mr(self._h, n.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), n.size,
                                               byref(t)))
        return t.value, n.size

    def wait(self, ticket: int, timeout_ms: int = 60_000) -> int:
        """0 when done, else the error code (-6 = timeout)."""
        return self.lib.voss_server_wait(self._h, ticket, timeout_ms)

    def result_interval(self, ticket: int) -> np.ndarray:
        out = np.zeros(1, dtype=INTERVAL_DTYPE)
        N.check(self.lib.voss_server_result_interval(self._h, ticket, out.ctypes.data_as(ctypes.POINTER(N.IntervalStats))))
        return out[0]

    def result_mr(self, ticket: int, count: int) -> np.ndarray:
        out = np.zeros(count, dtype=np.uint8)
        N.check(self.lib.voss_server_result_mr(self._h, ticket, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), count))
        return out

    def times(self, ticket: int) -> tuple[float, float, float]:
        a, b, c = c_double(), c_double(), c_double()
        N.check(self.lib.voss_server_request_times(self._h, ticket, byref(a), byref(b), byref(c)))
        return a.value, b.value, c.value

    def release(self, ticket: int) -> None:
        N.check(self.lib.voss_server_release(self._h, ticket))

    def stats(self) -> dict:
        s = N.ServerStats()
        N.check(self.lib.voss_server_get_stats(self._h, byref(s)))
        return {k: getattr(s, k) for k, _ in N.ServerStats._fields_ if not k.startswith("reserved")}


def request_stream(rate: float, count: int, seed: int = 20261203, mr_frac: float = 0.3,
                   start_exp=(9.0, 18.0), len_exp=(3.0, 9.0), mr_exp=(3.0, 6.0)):
    """A seeded Poisson arrival stream: (arrival_s, kind, payload) with kind 'iv' (lo, hi) or
    'mr' (uint64 array of odd values)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    out = []
    for i in range(count):
        if rng.random() < mr_frac:
            k = int(10 ** rng.uniform(*mr_exp))
            vals = rng.integers(0, 2**63, size=k, dtype=np.uint64) * 2 + 1
            out.append((float(t[i]), "mr", vals))
        else:
            lo = int(10 ** rng.uniform(*start_exp))
            ln = int(10 ** rng.uniform(*len_exp))
            out.append((float(t[i]), "iv", (lo, lo + ln)))
    return out


def serve_stream(server: Server, stream, collect: bool = False):
    """Submit each request at its arrival time (busy-waiting for precision) while a collector
    thread waits for completions; returns per-request latency (s) from the server's own clock
    and, if collect, the results."""
    tickets = [None] * len(stream)
    lat = np.full(len(stream), np.nan)
    results = [None] * len(stream) if collect else None
    submitted = threading.Semaphore(0)
    err = []

    def collector():
        for i in range(len(stream)):
            submitted.acquire()
            t, kind, count = tickets[i]
            rc = server.wait(t, 600_000)
            if rc != 0:
                err.append((i, rc))
                continue
            s, _, d = server.times(t)
            lat[i] = d - s
            if collect:
                results[i] = server.result_interval(t) if kind == "iv" else server.result_mr(t, count)
            server.release(t)

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for i, (at, kind, payload) in enumerate(stream):
        while time.perf_counter() - t0 < at:
            pass
        if kind == "iv":
            tickets[i] = (server.submit_interval(*payload), kind, 0)
        else:
            tk, cnt = server.submit_mr(payload)
            tickets[i] = (tk, kind, cnt)
        submitted.release()
    th.join()
    wall = time.perf_counter() - t0
    return lat, wall, results, err


def serve_plain(ctx: Context, stream, time_cap: float = float("inf")):
    """The same stream served one request at a time with one plain launch per request (no
    batching, no overlap), in arrival order, stopping after time_cap seconds.  Returns the
    latencies (completion - arrival) of the requests served and the elapsed time."""
    lat = []
    t0 = time.perf_counter()
    for at, kind, payload in stream:
        while time.perf_counter() - t0 < at:
            pass
        if kind == "iv":
            ctx.sieve_intervals(np.array([payload[0]], dtype=np.uint64), np.array([payload[1]], dtype=np.uint64))
        else:
            ctx.mr_verify(payload)
        done = time.perf_counter() - t0
        lat.append(done - at)
        if done > time_cap:
            break
    return np.array(lat), time.perf_counter() - t0

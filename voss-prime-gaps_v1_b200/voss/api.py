"""Python face of libvoss.so: a device context with the sieve, interval, Miller-Rabin and
gap-proof entry points, returning numpy arrays.

Every method calls straight into the C ABI; nothing here computes primes itself.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_int, c_uint32, c_uint64, c_void_p
from dataclasses import dataclass, field

import numpy as np

from . import _native as N


def _u64p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


@dataclass
class RangeResult:
    """Statistics of one range; arrays are numpy copies of voss_range_stats fields."""

    lo: int
    hi: int
    flags: int
    seg_num: int
    prime_count: int
    first_prime: int
    last_prime: int
    max_gap: int
    max_gap_lo: int
    mod4: np.ndarray
    modq: np.ndarray
    modq_gap: np.ndarray
    large_total: int
    gap_hist: np.ndarray
    large: np.ndarray = field(default_factory=lambda: np.zeros(0, dtype=LARGE_DTYPE))
    raw: N.RangeStats | None = None

    def modq_counts(self, q: int) -> np.ndarray:
        off = 0
        for qq in N.Q_LIST:
            if qq == q:
                return self.modq[off:off + q]
            off += qq
        raise KeyError(q)


LARGE_DTYPE = np.dtype([("position", "<u8"), ("gap", "<i4"), ("merit", "<f4")])


def range_result(st: N.RangeStats, large: np.ndarray | None = None) -> RangeResult:
    return RangeResult(
        lo=st.lo, hi=st.hi, flags=st.flags, seg_num=st.seg_num, prime_count=st.prime_count,
        first_prime=st.first_prime, last_prime=st.last_prime, max_gap=st.max_gap,
        max_gap_lo=st.max_gap_lo, mod4=np.ctypeslib.as_array(st.mod4).copy(),
        modq=np.ctypeslib.as_array(st.modq).copy(),
        modq_gap=np.ctypeslib.as_array(st.modq_gap).reshape(N.MODQ_ROWS, N.MODQ_MAX_GAP).copy(),
        large_total=st.large_total, gap_hist=np.ctypeslib.as_array(st.gap_hist).copy(),
        large=large if large is not None else np.zeros(0, dtype=LARGE_DTYPE), raw=st,
    )


INTERVAL_DTYPE = np.dtype([
    ("lo", "<u8"), ("hi", "<u8"), ("prime_count", "<u8"), ("first_prime", "<u8"), ("last_prime", "<u8"),
    ("max_gap", "<u8"), ("max_gap_lo", "<u8"), ("gap_overflow", "<u8"), ("gap_hist", "<u8", (N.IHIST,)),
])
assert INTERVAL_DTYPE.itemsize == ctypes.sizeof(N.IntervalStats)
assert LARGE_DTYPE.itemsize == ctypes.sizeof(N.LargeGap)


class Context:
    """A device context (voss_ctx_create): base primes up to isqrt(max_hi-1) resident on `device`."""

    def __init__(self, max_hi: int, device: int = 0, lib_path: str | None = None):
        self.lib = N.load(lib_path)
        h = c_void_p()
        N.check(self.lib.voss_ctx_create(device, max_hi, byref(h)))
        self._h = h
        self.device = device

    # -- lifetime ---------------------------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self.lib.voss_ctx_destroy(self._h)
            self._h = c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> c_void_p:
        return self._h

    def info(self) -> dict:
        mh, nb, sm = c_uint64(), c_uint64(), c_int()
        N.check(self.lib.voss_ctx_info(self._h, byref(mh), byref(nb), byref(sm)))
        return {"max_hi": mh.value, "base_primes": nb.value, "sm_count": sm.value}

    def tuning(self) -> dict:
        t = N.Tuning()
        N.check(self.lib.voss_ctx_get_tuning(self._h, byref(t)))
        return {k: getattr(t, k) for k in ("block_threads", "chunk_words", "ctas_per_sm", "coop_div", "mult_factor",
                                           "medium_mode", "walk_sixteenths", "mr_route")}

    def set_tuning(self, **kw) -> dict:
        t = N.Tuning()
        for k, v in kw.items():
            setattr(t, k, int(v))
        N.check(self.lib.voss_ctx_set_tuning(self._h, byref(t)))
        return self.tuning()

    def _large_buffer(self, cap: int) -> np.ndarray:
        """A reused output buffer for large-gap lists (only the written part is copied out), so
        that repeated calls touch no fresh pages."""
        buf = getattr(self, "_large_buf", None)
        if buf is None or buf.size < cap:
            buf = np.empty(max(cap, 1), dtype=LARGE_DTYPE)
            self._large_buf = buf
        return buf[:max(cap, 1)]

    # -- sieve ------------------------------------------------------------------------------
    def sieve_range(self, lo: int, hi: int, compat: bool = False, seg_num: int = 30_000_000_000,
                    large_cap: int = 1 << 22) -> RangeResult:
        st = N.RangeStats()
        large = self._large_buffer(large_cap)
        w = c_uint64()
        N.check(self.lib.voss_sieve_range(
            self._h, lo, hi, N.FLAG_REF_COMPAT if compat else 0, seg_num if compat else 0, byref(st),
            large.ctypes.data_as(ctypes.POINTER(N.LargeGap)), large_cap, byref(w)))
        return range_result(st, large[: w.value].copy())

    def sieve_range_device(self, lo: int, hi: int, compat: bool = False, seg_num: int = 30_000_000_000,
                           stream: int = 0) -> None:
        N.check(self.lib.voss_sieve_range_device(self._h, lo, hi, N.FLAG_REF_COMPAT if compat else 0,
                                                 seg_num if compat else 0, c_void_p(stream or None)))

    def fetch_range(self, large_cap: int = 1 << 22) -> RangeResult:
        st = N.RangeStats()
        large = self._large_buffer(large_cap)
        w = c_uint64()
        N.check(self.lib.voss_fetch_range(self._h, byref(st), large.ctypes.data_as(ctypes.POINTER(N.LargeGap)),
                                          large_cap, byref(w)))
        return range_result(st, large[: w.value].copy())

    def last_kernel_ms(self) -> tuple[float, float]:
        a, b = c_double(), c_double()
        N.check(self.lib.voss_last_kernel_ms(self._h, byref(a), byref(b)))
        return a.value, b.value

    def last_phase_ms(self) -> tuple[float, float, float, int]:
        """(pre-pass incl. copies and memsets, tile kernel, stitch/reduce/finalize) in ms of the
        last launch, and the number of kernels it launched."""
        a, b, t, k = c_double(), c_double(), c_double(), c_uint32()
        N.check(self.lib.voss_last_phase_ms(self._h, byref(a), byref(b), byref(t), byref(k)))
        return a.value, b.value, t.value, k.value

    def primes_range(self, lo: int, hi: int, cap: int | None = None) -> np.ndarray:
        cnt = c_uint64()
        if cap is None:
            N.check(self.lib.voss_primes_range(self._h, lo, hi, None, 0, byref(cnt)))
            cap = cnt.value
        out = np.zeros(max(cap, 1), dtype=np.uint64)
        N.check(self.lib.voss_primes_range(self._h, lo, hi, _u64p(out), cap, byref(cnt)))
        return out[: min(cap, cnt.value)]

    def gaps_at_least(self, lo: int, hi: int, min_gap: int, cap: int | None = None) -> np.ndarray:
        """All gaps >= min_gap in [lo, hi) as LARGE_DTYPE records (position = upper prime)."""
        cnt = c_uint64()
        if cap is None:
            cap = 1 << 20
        while True:
            out = np.empty(max(cap, 1), dtype=LARGE_DTYPE)
            N.check(self.lib.voss_gaps_at_least(self._h, lo, hi, min_gap,
                                                out.ctypes.data_as(ctypes.POINTER(N.LargeGap)), cap, byref(cnt)))
            if cnt.value <= cap:
                return out[: cnt.value].copy()
            cap = cnt.value

    def sieve_intervals(self, lo, hi) -> np.ndarray:
        lo = np.ascontiguousarray(lo, dtype=np.uint64)
        hi = np.ascontiguousarray(hi, dtype=np.uint64)
        if lo.shape != hi.shape:
            raise ValueError("lo and hi differ in shape")
        out = np.empty(lo.size, dtype=INTERVAL_DTYPE)  # every record is written by the call
        N.check(self.lib.voss_sieve_intervals(self._h, _u64p(lo), _u64p(hi), lo.size,
                                              out.ctypes.data_as(ctypes.POINTER(N.IntervalStats))))
        return out

    def gap_sequence(self, n: int, seg_num: int = 30_000_000_000, seq_size: int = 5_000_000):
        """voss_gap_sequence: the reference's sampled gap sequence of [1, n] (gap, lower prime)."""
        gap = np.zeros(seq_size, dtype=np.int32)
        p = np.zeros(seq_size, dtype=np.uint64)
        w = c_uint64()
        N.check(self.lib.voss_gap_sequence(self._h, n, seg_num, seq_size,
                                           gap.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _u64p(p), byref(w)))
        return gap, p

    def run_checkpointed(self, n: int, seg_num: int = 30_000_000_000, compat: bool = True, ckpt_every: int = 5,
                         directory: str = ".", large_cap: int = 1 << 22):
        """voss_run_checkpointed: [1, n] segment by segment with checkpoint.bin / stop.txt in
        `directory`.  Returns (RangeResult, resumed_from); raises VossError(-7) when stopped."""
        st = N.RangeStats()
        large = np.empty(large_cap, dtype=LARGE_DTYPE)  # only the written part is kept
        w, res = c_uint64(), c_uint64()
        N.check(self.lib.voss_run_checkpointed(self._h, n, seg_num, N.FLAG_REF_COMPAT if compat else 0, ckpt_every,
                                               directory.encode(), byref(st),
                                               large.ctypes.data_as(ctypes.POINTER(N.LargeGap)), large_cap,
                                               byref(w), byref(res)))
        return range_result(st, large[: w.value].copy()), res.value

    # -- Miller-Rabin / proofs --------------------------------------------------------------
    def mr_verify(self, n) -> np.ndarray:
        n = np.ascontiguousarray(n, dtype=np.uint64)
        out = np.zeros(n.size, dtype=np.uint8)
        N.check(self.lib.voss_mr_verify(self._h, _u64p(n), n.size,
                                        out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    def mr_verify_device(self, d_n: int, count: int, d_out: int, stream: int = 0) -> None:
        N.check(self.lib.voss_mr_verify_device(self._h, c_void_p(d_n), count, c_void_p(d_out),
                                               c_void_p(stream or None)))

    def prove_gaps(self, p_after, gap) -> np.ndarray:
        p = np.ascontiguousarray(p_after, dtype=np.uint64)
        g = np.ascontiguousarray(gap, dtype=np.int32)
        out = np.zeros(p.size, dtype=np.uint8)
        N.check(self.lib.voss_prove_gaps(self._h, _u64p(p), g.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                         p.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    def sha256_batch(self, messages) -> np.ndarray:
        """SHA-256 digests of a list of byte strings on the GPU, as a (len, 32) uint8 array."""
        msgs = [bytes(m) for m in messages]
        off = np.zeros(len(msgs) + 1, dtype=np.uint64)
        if msgs:
            off[1:] = np.cumsum([len(m) for m in msgs], dtype=np.uint64)
        data = np.frombuffer(b"".join(msgs), dtype=np.uint8) if off[-1] else np.zeros(1, dtype=np.uint8)
        out = np.zeros((len(msgs), 32), dtype=np.uint8)
        if msgs:
            N.check(self.lib.voss_sha256_batch(self._h, data.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), _u64p(off),
                                               len(msgs), out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out

    def probe_smem_rmw(self) -> float:
        g = c_double()
        N.check(self.lib.voss_probe_smem_rmw(self._h, byref(g)))
        return g.value

    def probe_mulmod(self) -> tuple[float, float]:
        """Montgomery products/s of this device for 64-bit moduli and for moduli below 2^63."""
        f, s = c_double(), c_double()
        N.check(self.lib.voss_probe_mulmod(self._h, byref(f), byref(s)))
        return f.value, s.value


def write_artifacts(res: RangeResult, out_dir: str) -> None:
    """Write the reference's CSV artifacts for a REF_COMPAT range (voss_write_artifacts)."""
    lib = N.load()
    large = np.ascontiguousarray(res.large, dtype=LARGE_DTYPE)
    st = res.raw if res.raw is not None else to_struct(res)
    N.check(lib.voss_write_artifacts(byref(st), large.ctypes.data_as(ctypes.POINTER(N.LargeGap)),
                                     large.size, out_dir.encode()))


def to_struct(res: RangeResult) -> N.RangeStats:
    st = N.RangeStats()
    for k in ("lo", "hi", "flags", "seg_num", "prime_count", "first_prime", "last_prime", "max_gap",
              "max_gap_lo", "large_total"):
        setattr(st, k, int(getattr(res, k)))
    np.ctypeslib.as_array(st.mod4)[:] = res.mod4
    np.ctypeslib.as_array(st.modq)[:] = res.modq
    np.ctypeslib.as_array(st.modq_gap)[:] = res.modq_gap
    np.ctypeslib.as_array(st.gap_hist)[:] = res.gap_hist
    return st


def merge_stats(parts: list[RangeResult], large_cap: int | None = None) -> RangeResult:
    """Combine adjacent-range results (voss_stats_merge): the host half of a sharded range."""
    lib = N.load()
    arr = (N.RangeStats * len(parts))()
    for i, p in enumerate(parts):
        arr[i] = p.raw if p.raw is not None else to_struct(p)
    large_in = np.concatenate([np.asarray(p.large, dtype=LARGE_DTYPE) for p in parts]) if parts else \
        np.zeros(0, dtype=LARGE_DTYPE)
    cap = large_cap if large_cap is not None else large_in.size + len(parts) + 1
    large = np.zeros(max(cap, 1), dtype=LARGE_DTYPE)
    large[: large_in.size] = large_in[:cap]
    out = N.RangeStats()
    w = c_uint64()
    N.check(lib.voss_stats_merge(arr, len(parts), byref(out), large.ctypes.data_as(ctypes.POINTER(N.LargeGap)),
                                 min(large_in.size, cap), cap, byref(w)))
    return range_result(out, large[: w.value].copy())


def write_gap_sequence(gap, p, out_dir: str) -> None:
    """voss_write_gap_sequence: gap_sequence.csv rows for the written entries."""
    gap = np.ascontiguousarray(gap, dtype=np.int32)
    p = np.ascontiguousarray(p, dtype=np.uint64)
    N.check(N.load().voss_write_gap_sequence(gap.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _u64p(p), gap.size,
                                             out_dir.encode()))


def run_checkpointed_fn(segment, n: int, seg_num: int, compat: bool, ckpt_every: int, directory: str,
                        large_cap: int = 1 << 22):
    """voss_run_checkpointed_fn over a Python segment function segment(lo, hi) -> RangeResult
    (any source of statistics: the device, or a CPU oracle in tests)."""
    lib = N.load()

    def cb(user, lo, hi, out, large, cap, written):
        try:
            r = segment(lo, hi)
            st = r.raw if r.raw is not None else to_struct(r)
            ctypes.memmove(out, ctypes.byref(st), ctypes.sizeof(N.RangeStats))
            k = min(cap, r.large.size)
            if k:
                ctypes.memmove(large, np.ascontiguousarray(r.large[:k]).ctypes.data, k * LARGE_DTYPE.itemsize)
            written[0] = k
            return 0
        except Exception:
            return -9

    fn = N.SEGMENT_FN(cb)
    st = N.RangeStats()
    large = np.empty(large_cap, dtype=LARGE_DTYPE)  # only the written part is kept
    w, res = c_uint64(), c_uint64()
    N.check(lib.voss_run_checkpointed_fn(fn, None, n, seg_num, N.FLAG_REF_COMPAT if compat else 0, ckpt_every,
                                         directory.encode(), byref(st),
                                         large.ctypes.data_as(ctypes.POINTER(N.LargeGap)), large_cap, byref(w),
                                         byref(res)))
    return range_result(st, large[: w.value].copy()), res.value


NOALLOC_MAX_COUNT = 1 << 22


def mr_verify_noalloc(d_n: int, count: int, d_is_prime: int, stream: int = 0) -> None:
    """voss_mr_verify_noalloc: Miller-Rabin verdicts into device memory without allocating
    anything (no context; scratch is a fixed array inside the library, at most
    NOALLOC_MAX_COUNT candidates per call, calls must not overlap on the GPU)."""
    N.check(N.load().voss_mr_verify_noalloc(c_void_p(d_n), count, c_void_p(d_is_prime), c_void_p(stream or None)))


def device_count() -> int:
    n = c_int()
    N.check(N.load().voss_device_count(byref(n)))
    return n.value


def version() -> str:
    return N.load().voss_version().decode()

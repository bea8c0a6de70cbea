"""The C ABI of libvoss.so on the CPU: every declared symbol is exported, the ctypes mirrors
match the C layouts, errors are reported instead of exiting, and the two host-only entry
points (voss_write_artifacts, voss_stats_merge) are checked against independent statements
of the reference's rules.  No compute call needs a GPU here."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle_lib as O
import voss
from voss import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "voss.h")
SEG = 30_000_000_000


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"VOSS_API\s+[\w\s\*]+?\b(voss_\w+)\s*\(", txt)))


def test_every_declared_symbol_is_exported_and_bound():
    names = declared_functions()
    assert len(names) >= 20
    lib = N.load()
    for n in names:
        assert hasattr(lib, n), n
        assert n in N.SIGNATURES, f"{n} has no ctypes signature"
    out = subprocess.run(["nm", "-D", "--defined-only", N.lib_path()], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (voss_\w+)", out))
    assert set(names) <= exported


def test_struct_layouts_match_c():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "voss.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(voss_range_stats), sizeof(voss_interval_stats), sizeof(voss_large_gap), sizeof(voss_tuning));
  printf("%zu %zu %zu %zu %zu\n", offsetof(voss_range_stats, mod4), offsetof(voss_range_stats, modq),
         offsetof(voss_range_stats, modq_gap), offsetof(voss_range_stats, large_total), offsetof(voss_range_stats, gap_hist));
  printf("%zu %zu\n", offsetof(voss_interval_stats, gap_overflow), offsetof(voss_interval_stats, gap_hist));
  printf("%zu %zu %zu %zu\n", sizeof(voss_server_config), offsetof(voss_server_config, max_batch_candidates),
         sizeof(voss_server_stats), offsetof(voss_server_stats, mean_batch_requests));
  return 0;
}'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        nums = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    RS, IS = N.RangeStats, N.IntervalStats
    assert nums[:4] == [ctypes.sizeof(RS), ctypes.sizeof(IS), ctypes.sizeof(N.LargeGap), ctypes.sizeof(N.Tuning)]
    assert nums[4:9] == [RS.mod4.offset, RS.modq.offset, RS.modq_gap.offset, RS.large_total.offset, RS.gap_hist.offset]
    assert nums[9:11] == [IS.gap_overflow.offset, IS.gap_hist.offset]
    SC, SS = N.ServerConfig, N.ServerStats
    assert nums[11:15] == [ctypes.sizeof(SC), SC.max_batch_candidates.offset, ctypes.sizeof(SS),
                           SS.mean_batch_requests.offset]


def test_errors_are_returned_not_fatal():
    lib = N.load()
    h = ctypes.c_void_p()
    rc = lib.voss_ctx_create(0, 7, ctypes.byref(h))      # max_hi below the minimum
    assert rc == -1 and b"max_hi" in lib.voss_last_error()
    rc = lib.voss_ctx_create(0, 10**9, None)
    assert rc == -1
    if voss.device_count() == 0:
        rc = lib.voss_ctx_create(0, 10**9, ctypes.byref(h))
        assert rc == -10 and b"no CUDA device" in lib.voss_last_error()
        with pytest.raises(voss.VossError):
            voss.Context(10**9)
    assert lib.voss_mr_verify_noalloc(None, 3, None, None) == -1


# ---- artifacts -------------------------------------------------------------------------
def reference_format_csvs(r, large):
    """The reference's writers (voss_v7_live.cu:707-827) restated with Python formatting."""
    N_ = r.hi - 1
    g = r.gap_hist
    out = {}
    out["gap_histogram.csv"] = "gap,count\n" + "".join(f"{i},{int(g[i])}\n" for i in range(1, 100000) if g[i] > 0)
    hl = [(1000000000, 1.7783), (10000000000, 1.8018), (100000000000, 1.8208), (1000000000000, 1.8366),
          (10000000000000, 1.8497)]
    s = "N,P6_over_P2\n" + "".join(f"{n},{v:.6f}\n" for n, v in hl)
    if N_ not in [n for n, _ in hl]:
        s += f"{N_},{float(g[6]) / float(g[2]):.6f}\n"
    out["hl_trend.csv"] = s
    s = "q,a,count\n"
    for q in (6, 30):
        c = r.modq_counts(q)
        s += "".join(f"{q},{a},{int(c[a])}\n" for a in range(q))
    out["modq_counts.csv"] = s
    s = "q,residue,gap,count\n"
    rows = [(6, [1, 5], 0), (30, [1, 7, 11, 13, 17, 19, 23, 29], 2)]
    for q, res, off in rows:
        for ri, rr in enumerate(res):
            for gg in range(1, 100):
                c = int(r.modq_gap[off + ri, gg])
                if c > 0:
                    s += f"{q},{rr},{gg},{c}\n"
    out["modq_gap_hist.csv"] = s
    p41, p43 = int(r.mod4[0]), int(r.mod4[1])
    out["chebyshev.csv"] = f"N,pi_4_1,pi_4_3,difference\n{N_},{p41},{p43},{p43 - p41}\n"
    order = sorted(range(large.size), key=lambda i: (-float(large["merit"][i]), int(large["position"][i])))
    out["large_gaps.csv"] = "position,gap,merit\n" + "".join(
        f"{int(large['position'][i])},{int(large['gap'][i])},{float(large['merit'][i]):.6f}\n" for i in order)
    return out


@pytest.mark.parametrize("n", [10**4, 10**7])
def test_write_artifacts_byte_format(n):
    r = O.sieve_range(1, n + 1, compat=True, seg_num=SEG)
    with tempfile.TemporaryDirectory() as d:
        voss.write_artifacts(r, d)
        want = reference_format_csvs(r, r.large)
        for name, text in want.items():
            assert open(os.path.join(d, name)).read() == text, name


def test_write_artifacts_reports_io_error():
    r = O.sieve_range(1, 1001, compat=True, seg_num=SEG)
    with pytest.raises(voss.VossError) as e:
        voss.write_artifacts(r, "/nonexistent/dir")
    assert e.value.code == -8


# ---- sharded-range merge ----------------------------------------------------------------
def assert_same(a, b):
    for k in ("lo", "hi", "prime_count", "first_prime", "last_prime", "max_gap", "max_gap_lo", "large_total"):
        assert getattr(a, k) == getattr(b, k), k
    for k in ("mod4", "modq", "modq_gap", "gap_hist"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)
    assert sorted(zip(a.large["position"].tolist(), a.large["gap"].tolist())) == \
        sorted(zip(b.large["position"].tolist(), b.large["gap"].tolist()))


@pytest.mark.parametrize("compat,seg", [(True, SEG), (True, 2_000_010), (False, 0)])
def test_merge_of_parts_equals_whole(compat, seg):
    cuts = [1, 5, 6, 1000, 3_000_007, 9_999_991, 20_000_001]
    parts = [O.sieve_range(a, b, compat=compat, seg_num=seg) for a, b in zip(cuts, cuts[1:])]
    whole = O.sieve_range(cuts[0], cuts[-1], compat=compat, seg_num=seg)
    assert_same(voss.merge_stats(parts), whole)


def _gloo_rank(rank, world, port, out_path):
    import pickle

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    n = 4_000_000
    lo, hi = rank * n + 1, (rank + 1) * n + 1
    r = O.sieve_range(lo, hi, compat=True, seg_num=SEG)   # stands in for this rank's GPU sieve
    blob = (bytes(voss.to_struct(r)), r.large.tobytes())
    got = [None] * world
    dist.all_gather_object(got, blob)
    if rank == 0:
        parts = []
        for sb, lb in got:
            st = N.RangeStats.from_buffer_copy(sb)
            parts.append(voss.range_result(st, np.frombuffer(lb, dtype=voss.LARGE_DTYPE).copy()))
        m = voss.merge_stats(parts)
        pickle.dump((bytes(voss.to_struct(m)), m.large.tobytes()), open(out_path, "wb"))
    dist.destroy_process_group()


def test_two_rank_gloo_merge_equals_single_range():
    import pickle
    import socket

    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "m.pkl")
        mp.spawn(_gloo_rank, args=(2, port, out), nprocs=2, join=True)
        sb, lb = pickle.load(open(out, "rb"))
    m = voss.range_result(N.RangeStats.from_buffer_copy(sb), np.frombuffer(lb, dtype=voss.LARGE_DTYPE).copy())
    whole = O.sieve_range(1, 8_000_001, compat=True, seg_num=SEG)
    assert_same(m, whole)

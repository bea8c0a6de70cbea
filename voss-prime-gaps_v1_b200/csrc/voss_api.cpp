// voss_api.cpp — host runtime and C ABI of libvoss.so (declared in include/voss.h).
//
// Replaces the host half of src/voss_v7_live.cu main() (:337-837): base-prime generation
// (:96-118), the segment loop's launch-list building and host accumulation (:434-626), the
// epilogue statistics (:634-705) and the CSV writers (:707-827); and the driver half of
// src/verify_cpp.cpp main() (:112-276) for batch Miller-Rabin and gap proofs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cinttypes>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "voss.h"
#include "voss_internal.h"
#include "voss_host.h"

using namespace voss;

namespace voss_host {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int DevBuf::ensure(size_t need) {
  if (need <= bytes) return VOSS_OK;
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  size_t n = need < 256 ? 256 : need + need / 4;
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    p = nullptr;
    return fail(VOSS_ERR_NOMEM, "cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
  }
  bytes = n;
  return VOSS_OK;
}

const int kW30[8] = {1, 7, 11, 13, 17, 19, 23, 29};
const int kQ[VOSS_NUM_Q] = VOSS_Q_LIST;

// Wheel integers (coprime to 30) below x within its block of 30, and below x in all.
constexpr uint8_t kCoprime30Below[30] = {0, 0, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 4,
                                         4, 4, 4, 5, 5, 6, 6, 6, 6, 7, 7, 7, 7, 7, 7};
uint64_t wheel_count_below(uint64_t x) { return 8ull * (x / 30) + kCoprime30Below[x % 30]; }

uint64_t isqrt_u64(uint64_t x) {
  uint64_t s = (uint64_t)std::sqrt((long double)x);
  while (s * s > x) --s;
  while ((s + 1) * (s + 1) <= x) ++s;
  return s;
}

// Primes 37 <= p <= limit, by an odd-only segmented sieve.
std::vector<uint32_t> base_primes(uint64_t limit) {
  std::vector<uint32_t> out;
  if (limit < 37) return out;
  const uint64_t r = isqrt_u64(limit);
  std::vector<uint8_t> small(r + 1, 1);
  std::vector<uint32_t> sp;
  for (uint64_t i = 2; i <= r; ++i) {
    if (!small[i]) continue;
    sp.push_back((uint32_t)i);
    for (uint64_t j = i * i; j <= r; j += i) small[j] = 0;
  }
  out.reserve((size_t)(limit / (std::log((double)limit) - 1.1)) + 16);
  const uint64_t SEG = 1u << 21;  // odd slots per segment
  std::vector<uint8_t> seg(SEG);
  for (uint64_t base = 0; base <= limit; base += 2 * SEG) {
    // slot i <-> value base + 2i + 1
    std::fill(seg.begin(), seg.end(), 1);
    const uint64_t vmax = std::min(limit, base + 2 * SEG - 1);
    for (uint32_t q : sp) {
      if (q == 2) continue;
      const uint64_t qq = (uint64_t)q * q;
      if (qq > vmax) break;
      uint64_t m = std::max(qq, (base + 1 + q - 1) / q * q);
      if ((m & 1) == 0) m += q;
      for (uint64_t i = (m - base - 1) / 2; i < SEG; i += q) seg[i] = 0;
    }
    for (uint64_t i = 0; i < SEG; ++i) {
      const uint64_t v = base + 2 * i + 1;
      if (v > vmax) break;
      if (seg[i] && v >= 37) out.push_back((uint32_t)v);
    }
  }
  return out;
}


}  // namespace

namespace voss_detail {
int set_error(int code, const char* msg) { return voss_host::fail(code, "%s", msg); }
}  // namespace voss_detail


namespace voss_host {

int apply_tuning(voss_ctx* c, const voss_tuning& t0) {
  voss_tuning t = t0;
  if (!t.block_threads) t.block_threads = 1024;
  if (!t.chunk_words) t.chunk_words = t.block_threads == 1024 ? 49 : 45;
  if (!t.coop_div) t.coop_div = 80;
  if (!t.mult_factor) t.mult_factor = 8;
  if (!t.walk_sixteenths) t.walk_sixteenths = 4;
  if (!t.mr_route) t.mr_route = 50;
  if (t.block_threads != 512 && t.block_threads != 1024)
    return fail(VOSS_ERR_ARG, "block_threads must be 512 or 1024");
  if (t.medium_mode > 1) return fail(VOSS_ERR_ARG, "medium_mode must be 0 or 1");
  // medium primes (p < mult_factor * tile bytes <= 64 * 1,044,480) keep 7p below 2^32 in the
  // 32-bit offset arithmetic of their clearing loops
  if (t.mult_factor > 64) return fail(VOSS_ERR_ARG, "mult_factor must be <= 64");
  if ((t.chunk_words & 1u) == 0 || t.chunk_words > 255)
    return fail(VOSS_ERR_ARG, "chunk_words must be odd and <= 255");
  const uint32_t tw = t.block_threads * t.chunk_words;
  // the tile kernel counts residue classes over the words w = c (mod 1001) of a tile in 6-bit
  // column counters: at most 63 such words (shared memory caps tiles near 52,000 words anyway)
  if (tw > 63u * 1001u) return fail(VOSS_ERR_ARG, "tile of %u words exceeds 63063 words", tw);
  const size_t smem = sieve_smem_bytes(tw);
  int maxc = 0;
  cudaSetDevice(c->device);
  if (sieve_kernel_attrs((int)t.block_threads, smem, &maxc) != 0 || maxc < 1)
    return fail(VOSS_ERR_ARG, "tile of %u words does not fit in shared memory (%zu bytes)", tw, smem);
  if (!t.ctas_per_sm || (int)t.ctas_per_sm > maxc) t.ctas_per_sm = (uint32_t)maxc;
  c->tune = t;
  c->ctas_per_sm = (int)t.ctas_per_sm;
  return VOSS_OK;
}


// Cut intervals [lo_i, hi_i) into tiles; intervals without wheel integers get no tiles.
int plan_intervals(const voss_ctx* c, const uint64_t* lo, const uint64_t* hi, uint32_t n,
                   uint64_t seg_k, RunPlan* P) {
  const uint64_t tw = (uint64_t)c->tune.block_threads * c->tune.chunk_words;
  P->iv.resize(n);
  uint64_t tiles = 0, words = 0;
  for (uint32_t i = 0; i < n; ++i) {
    IntervalDev& d = P->iv[i];
    std::memset(&d, 0, sizeof(d));
    const uint64_t a = std::max<uint64_t>(lo[i], 7);
    d.lo = a;
    d.hi = hi[i];
    d.seg_k = seg_k;
    d.tile_begin = (uint32_t)tiles;
    if (a >= hi[i]) {
      d.k0 = 0;
      d.n_words = 0;
      d.n_tiles = 0;
      continue;
    }
    const uint64_t kf = a / 30, kl = (hi[i] - 1) / 30;
    d.k0 = kf & ~3ull;
    d.n_words = (kl - d.k0) / 4 + 1;
    d.gword = words;
    words += d.n_words;
    const uint64_t nt = (d.n_words + tw - 1) / tw;
    d.n_tiles = (uint32_t)nt;
    tiles += nt;
    if (tiles >= 0x7FFFFFFFull) return fail(VOSS_ERR_RANGE, "too many tiles in one launch; split the range");
  }
  P->n_tiles = (uint32_t)tiles;
  P->n_words = words;
  return VOSS_OK;
}


int launch_plan_ws(voss_ctx* c, Workspace& W, const LaunchEvents& E, const RunPlan& P, bool want_large,
                   uint64_t large_cap, bool emit, cudaStream_t s, uint32_t min_gap, SieveArgs* args_out) {
  const uint32_t n_iv = (uint32_t)P.iv.size();
  int rc;
  if ((rc = W.iv.ensure(sizeof(IntervalDev) * std::max<size_t>(1, n_iv)))) return rc;
  if ((rc = W.partials.ensure(sizeof(TilePartial) * std::max<size_t>(1, P.n_tiles)))) return rc;
  if ((rc = W.acc.ensure(sizeof(unsigned long long) * kAccStride * std::max<size_t>(1, n_iv)))) return rc;
  if ((rc = W.out.ensure(sizeof(IntervalOut) * std::max<size_t>(1, n_iv)))) return rc;
  if ((rc = W.counters.ensure(sizeof(uint32_t) * kCtrWords))) return rc;
  if ((rc = W.over.ensure(sizeof(OverflowGap) * kOverCap))) return rc;
  const uint64_t cap = want_large ? std::min(std::max(large_cap, (uint64_t)1), kMaxLargeCap) : 1;
  if ((rc = W.large.ensure(sizeof(LargeGapDev) * cap))) return rc;
  if ((rc = W.large_iv.ensure(sizeof(uint32_t) * cap))) return rc;

  SieveArgs a;
  std::memset(&a, 0, sizeof(a));
  a.primes = c->d_primes.as<uint32_t>();
  a.magic = c->d_magic.as<uint64_t>();
  a.n_primes = (uint32_t)c->primes.size();
  a.p_max = c->primes.empty() ? 0u : c->primes.back();
  a.pretab = c->d_pretab.as<uint32_t>();
  a.iv = W.iv.as<IntervalDev>();
  a.n_intervals = n_iv;
  a.n_tiles = P.n_tiles;
  a.tile_words = c->tune.block_threads * c->tune.chunk_words;
  a.chunk_words = c->tune.chunk_words;
  a.coop_div = c->tune.coop_div;
  a.mult_factor = c->tune.mult_factor;
  a.walk_sixteenths = c->tune.walk_sixteenths;
  a.want_large = want_large ? 1u : 0u;
  a.large_min_gap = min_gap;
  a.b_mode = c->tune.medium_mode;
  uint32_t* ctr = W.counters.as<uint32_t>();
  a.tile_counter = ctr + kCtrTile;
  a.large_count = ctr + kCtrLarge;
  a.over_count = ctr + kCtrOver;
  a.error = ctr + kCtrError;
  a.partials = W.partials.as<TilePartial>();
  a.acc = W.acc.as<unsigned long long>();
  a.large = W.large.as<LargeGapDev>();
  a.large_iv = W.large_iv.as<uint32_t>();
  a.large_cap = (uint32_t)cap;
  a.over = W.over.as<OverflowGap>();
  a.over_cap = kOverCap;
  if (emit) {
    a.tile_offset = W.offsets.as<unsigned long long>();
    a.out = W.emit.as<unsigned long long>();
    a.out_cap = W.emit.bytes / sizeof(unsigned long long);
  }
  const uint32_t tw = a.tile_words;
  const size_t smem = sieve_smem_bytes(tw);
  const int slots = c->sm_count * c->ctas_per_sm;
  const int grid = (int)std::max<uint32_t>(1, std::min<uint32_t>(P.n_tiles, (uint32_t)slots));
  // Large-prime pre-pass: primes p >= mult_factor * tile bytes are applied once per launch
  // (prime-major) instead of once per tile, when the launch's bitmap fits the budget.
  const uint64_t p_large = (uint64_t)c->tune.mult_factor * 4ull * tw;
  uint64_t max_sq = 0;
  for (const IntervalDev& d : P.iv)
    if (d.n_tiles) max_sq = std::max<uint64_t>(max_sq, isqrt_u64(d.hi - 1));
  const uint32_t j0 = (uint32_t)(std::lower_bound(c->primes.begin(), c->primes.end(), p_large) - c->primes.begin());
  const uint32_t j1 = (uint32_t)(std::upper_bound(c->primes.begin(), c->primes.end(),
                                                  (uint32_t)std::min<uint64_t>(max_sq, 0xFFFFFFFFull)) -
                                 c->primes.begin());
  const size_t gbm_bytes = (size_t)P.n_words * 4;
  bool scatter = P.n_tiles && j1 > j0 && p_large <= 0xFFFFFFFFull && gbm_bytes <= W.gbm_budget &&
                 (!W.gbm_fixed || gbm_bytes <= W.gbm.bytes);
  std::vector<IntervalScatter> sc;
  // Windows of consecutive intervals whose bitmap words total at most kScatterWindowBytes: the
  // pre-pass runs window by window, so that its atomics find their lines in L2 (the bitmap of a
  // whole launch can be gigabytes).  Inside a window, intervals are sorted by isqrt(hi)
  // descending (the kernel stops a prime at the first interval it does not reach).
  struct Window {
    uint32_t off, n, j1;
  };
  std::vector<Window> wins;
  if (scatter) {
    uint64_t wbytes = 0;
    for (const IntervalDev& d : P.iv) {
      if (!d.n_tiles) continue;
      const uint64_t sq = isqrt_u64(d.hi - 1);
      if (sq < p_large) continue;
      if (wins.empty() || (wbytes && wbytes + 4ull * d.n_words > kScatterWindowBytes)) {
        wins.push_back(Window{(uint32_t)sc.size(), 0, j0});
        wbytes = 0;
      }
      IntervalScatter I;
      I.vbase = 30ull * d.k0;
      I.span = 120ull * d.n_words;
      I.gword = d.gword;
      I.sqrt_hi = (uint32_t)std::min<uint64_t>(sq, 0xFFFFFFFFull);
      I.vbase_d = (double)I.vbase;
      I.vbase_lo = (uint32_t)I.vbase;
      I.span32 = (uint32_t)std::min<uint64_t>(I.span, 0xFFFFFFFFull);
      I.lt32 = I.span / 30 < (1ull << 31) ? (uint32_t)(I.span / 30) : 0u;
      sc.push_back(I);
      wbytes += 4ull * d.n_words;
      wins.back().n++;
    }
    for (Window& w : wins) {
      std::sort(sc.begin() + w.off, sc.begin() + w.off + w.n,
                [](const IntervalScatter& x, const IntervalScatter& y) { return x.sqrt_hi > y.sqrt_hi; });
      w.j1 = (uint32_t)(std::upper_bound(c->primes.begin(), c->primes.end(), sc[w.off].sqrt_hi) - c->primes.begin());
    }
    if ((rc = W.gbm.ensure(gbm_bytes)) || (rc = W.scat.ensure(sizeof(IntervalScatter) * sc.size()))) return rc;
    a.gbm = W.gbm.as<uint32_t>();
    a.scatter_first = j0;
  }
  // Tiles of a launch of many intervals find their interval in a table (one load) rather than
  // by a binary search of the interval descriptors in the tile header.
  std::vector<uint32_t> tiv;
  if (n_iv > 1 && P.n_tiles) {
    tiv.resize(P.n_tiles);
    for (uint32_t i = 0; i < n_iv; ++i)
      for (uint32_t t = 0; t < P.iv[i].n_tiles; ++t) tiv[P.iv[i].tile_begin + t] = i;
    if ((rc = W.tile_iv.ensure(sizeof(uint32_t) * P.n_tiles))) return rc;
    a.tile_iv = W.tile_iv.as<uint32_t>();
  }
  // Device work of the launch, all of it after ev0 (the host planning above is done first, so
  // the GPU never waits on the host inside the events).
  CUDA_TRY(cudaEventRecord(E.ev0, s));
  if (n_iv) CUDA_TRY(cudaMemcpyAsync(W.iv.p, P.iv.data(), sizeof(IntervalDev) * n_iv, cudaMemcpyHostToDevice, s));
  if (!tiv.empty())
    CUDA_TRY(cudaMemcpyAsync(W.tile_iv.p, tiv.data(), sizeof(uint32_t) * tiv.size(), cudaMemcpyHostToDevice, s));
  if (!emit) CUDA_TRY(cudaMemsetAsync(W.acc.p, 0, sizeof(unsigned long long) * kAccStride * std::max<size_t>(1, n_iv), s));
  CUDA_TRY(cudaMemsetAsync(W.counters.p, 0, sizeof(uint32_t) * kCtrWords, s));
  if (scatter) {
    CUDA_TRY(cudaMemsetAsync(W.gbm.p, 0xFF, gbm_bytes, s));
    CUDA_TRY(cudaMemcpyAsync(W.scat.p, sc.data(), sizeof(IntervalScatter) * sc.size(), cudaMemcpyHostToDevice, s));
  }
  for (const Window& w : wins)
    if (launch_scatter_large(a.primes, a.magic, j0, w.j1, W.scat.as<IntervalScatter>() + w.off, w.n,
                             W.gbm.as<uint32_t>(), c->sm_count, s))
      return fail(VOSS_ERR_CUDA, "large-prime pre-pass launch failed");
  if (E.evp) CUDA_TRY(cudaEventRecord(E.evp, s));
  if (P.n_tiles) {
    int lr = emit ? launch_sieve_emit(a, grid, (int)c->tune.block_threads, smem, s)
                  : launch_sieve_stats(a, grid, (int)c->tune.block_threads, smem, s);
    if (lr) return fail(VOSS_ERR_CUDA, "sieve launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  CUDA_TRY(cudaEventRecord(E.ev1, s));
  if (!emit) {
    if (launch_stitch(a, s)) return fail(VOSS_ERR_CUDA, "stitch launch failed");
    if (launch_reduce(a, W.out.as<IntervalOut>(), s)) return fail(VOSS_ERR_CUDA, "reduce launch failed");
  }
  CUDA_TRY(cudaEventRecord(E.ev2, s));
  if (&W == &c->ws)  // the context's own launches (server slots keep their own workspaces)
    c->last_kernels = (uint32_t)wins.size() + (P.n_tiles ? 1u : 0u) + (emit ? 0u : 2u);
  if (args_out) *args_out = a;
  return VOSS_OK;
}

int launch_plan(voss_ctx* c, const RunPlan& P, bool want_large, uint64_t large_cap, bool emit, cudaStream_t s,
                uint32_t min_gap = 0, SieveArgs* args_out = nullptr) {
  LaunchEvents E;
  E.ev0 = c->ev0;
  E.evp = c->evp;
  E.ev1 = c->ev1;
  E.ev2 = c->ev2;
  return launch_plan_ws(c, c->ws, E, P, want_large, large_cap, emit, s, min_gap, args_out);
}

// memcpy split over host threads: one thread copies from pageable memory at a fraction of the
// host's memory bandwidth.  A part whose thread cannot be started is copied by the caller.
void parallel_copy(void* dst, const void* src, size_t bytes, size_t min_part) {
  const size_t kMinPart = min_part;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t parts = std::min<size_t>({(size_t)std::min(hw, 8u), bytes / kMinPart + 1});
  if (parts <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const size_t step = (bytes / parts + 63) & ~(size_t)63;
  std::vector<std::thread> th;
  th.reserve(parts);
  for (size_t i = 1; i < parts; ++i) {
    const size_t a = std::min(bytes, i * step), b = std::min(bytes, (i + 1) * step);
    if (a >= b) continue;
    try {
      th.emplace_back([=] { std::memcpy((char*)dst + a, (const char*)src + a, b - a); });
    } catch (const std::exception&) {
      std::memcpy((char*)dst + a, (const char*)src + a, b - a);
    }
  }
  std::memcpy(dst, src, std::min(bytes, step));
  for (auto& t : th) t.join();
}

// Copies the segments one after another into dst, the concatenated bytes split evenly over up to
// 8 host threads (parts of at least min_part bytes).  A part whose thread cannot be started is
// copied by the caller.
void parallel_gather(void* dst, const CopySeg* seg, size_t n_seg, size_t min_part) {
  size_t total = 0;
  for (size_t i = 0; i < n_seg; ++i) total += seg[i].bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t parts = std::min<size_t>({(size_t)std::min(hw, 8u), total / std::max<size_t>(min_part, 1) + 1});
  auto copy_range = [=](size_t a, size_t b) {  // bytes [a, b) of the concatenation
    size_t pos = 0;
    for (size_t i = 0; i < n_seg && pos < b; ++i) {
      const size_t s0 = pos, s1 = pos + seg[i].bytes;
      pos = s1;
      const size_t x = std::max(a, s0), y = std::min(b, s1);
      if (x < y) std::memcpy((char*)dst + x, (const char*)seg[i].src + (x - s0), y - x);
    }
  };
  if (parts <= 1) {
    copy_range(0, total);
    return;
  }
  const size_t step = (total / parts + 63) & ~(size_t)63;
  std::vector<std::thread> th;
  th.reserve(parts);
  for (size_t i = 1; i < parts; ++i) {
    const size_t a = std::min(total, i * step), b = std::min(total, (i + 1) * step);
    if (a >= b) continue;
    try {
      th.emplace_back(copy_range, a, b);
    } catch (const std::exception&) {
      copy_range(a, b);
    }
  }
  copy_range(0, std::min(total, step));
  for (auto& t : th) t.join();
}

// The context's two pinned staging buffers, ready for host writes: every transfer that may
// still use them (left queued by an earlier call that returned early) has finished.  They hold
// min(entries, stage_limit) 64-bit words each (grow-only); callers move data in chunks of
// h_stage_cap words.
int ensure_stage(voss_ctx* c, size_t entries) {
  entries = std::max<size_t>(1, std::min(entries, c->stage_limit));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
  for (int b = 0; b < 2; ++b) CUDA_TRY(cudaEventSynchronize(c->ev_stage[b]));
  if (entries <= c->h_stage_cap) return VOSS_OK;
  for (int b = 0; b < 2; ++b) {
    if (c->h_stage[b]) cudaFreeHost(c->h_stage[b]);
    c->h_stage[b] = nullptr;
  }
  c->h_stage_cap = 0;
  for (int b = 0; b < 2; ++b)
    if (cudaMallocHost(&c->h_stage[b], entries * sizeof(uint64_t)) != cudaSuccess) {
      c->h_stage[b] = nullptr;
      return fail(VOSS_ERR_NOMEM, "cudaMallocHost of the staging buffers failed");
    }
  c->h_stage_cap = entries;
  return VOSS_OK;
}

// Host -> device through the staging buffers on stream s: chunk i is filled by host threads
// into buffer i & 1 once that buffer's previous transfer is done, then crosses while chunk
// i + 1 is filled.  Returns once the last chunk is queued.
int stage_in(voss_ctx* c, void* d_dst, const void* src, size_t bytes, cudaStream_t s) {
  const size_t chunk = c->h_stage_cap * sizeof(uint64_t);
  size_t i = 0;
  for (size_t off = 0; off < bytes; off += chunk, ++i) {
    const size_t k = std::min(chunk, bytes - off);
    const int b = (int)(i & 1);
    CUDA_TRY(cudaEventSynchronize(c->ev_stage[b]));
    parallel_copy(c->h_stage[b], (const char*)src + off, k);
    CUDA_TRY(cudaMemcpyAsync((char*)d_dst + off, c->h_stage[b], k, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaEventRecord(c->ev_stage[b], s));
  }
  return VOSS_OK;
}

// Device -> host through the staging buffers, after the work queued on s: chunk j crosses into
// buffer j & 1 while host threads copy chunk j - 1 out.  Returns with every byte in dst.
int stage_out(voss_ctx* c, void* dst, const void* d_src, size_t bytes, cudaStream_t s) {
  const size_t chunk = c->h_stage_cap * sizeof(uint64_t);
  size_t prev_off = 0, prev_k = 0, j = 0;
  for (size_t off = 0; off < bytes; off += chunk, ++j) {
    const size_t k = std::min(chunk, bytes - off);
    const int b = (int)(j & 1);
    CUDA_TRY(cudaEventSynchronize(c->ev_stage[b]));  // nothing of this buffer is still crossing in
    CUDA_TRY(cudaMemcpyAsync(c->h_stage[b], (const char*)d_src + off, k, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaEventRecord(c->ev_stage[b], s));
    if (j > 0) {
      CUDA_TRY(cudaEventSynchronize(c->ev_stage[b ^ 1]));
      parallel_copy((char*)dst + prev_off, c->h_stage[b ^ 1], prev_k);
    }
    prev_off = off;
    prev_k = k;
  }
  if (j > 0) {
    CUDA_TRY(cudaEventSynchronize(c->ev_stage[(j - 1) & 1]));
    parallel_copy((char*)dst + prev_off, c->h_stage[(j - 1) & 1], prev_k);
  }
  return VOSS_OK;
}

// Route a batch of intervals (see voss_host.h) and launch it.
void route_intervals(const voss_ctx* c, const uint64_t* lo, const uint64_t* hi, uint32_t n, uint64_t cand_cap,
                     IntervalRoute* R) {
  NvtxRange r("route");
  // An interval whose base primes outnumber mr_route times its length costs more in per-prime
  // reductions (one per prime in the pre-pass or in its tiles: a short interval is one partial
  // tile, for which every prime above 8 tile lengths is a "large" prime) than Miller-Rabin of
  // its wheel integers costs; it goes to short_iv.cu.
  const uint64_t route = c->tune.mr_route;
  for (uint32_t i = 0; i < n; ++i) {
    const uint64_t a = std::max<uint64_t>(lo[i], 7);
    bool mr = false;
    if (route != 0xFFFFFFFFull && a < hi[i]) {
      const uint64_t sq = isqrt_u64(hi[i] - 1);
      const size_t np = (size_t)(std::upper_bound(c->primes.begin(), c->primes.end(),
                                                  (uint32_t)std::min<uint64_t>(sq, 0xFFFFFFFFull)) -
                                 c->primes.begin());
      const uint64_t pairs = np;
      const uint64_t len = hi[i] - a;
      mr = len < (1ull << 31) && pairs / route > len && R->n_cand + len <= cand_cap;
    }
    if (mr) {
      ShortInterval I;
      I.base = 30ull * (a / 30);
      I.cand_off = R->n_cand;
      I.j0 = (uint32_t)kCoprime30Below[a % 30];
      I.n_cand = (uint32_t)(wheel_count_below(hi[i]) - wheel_count_below(a));
      I.out_index = i;
      I.pad = 0;
      R->n_cand += I.n_cand;
      R->sv.push_back(I);
    } else {
      R->lo.push_back(lo[i]);
      R->hi.push_back(hi[i]);
      R->map.push_back(i);
    }
  }
}

int launch_routed(voss_ctx* c, Workspace& W, const LaunchEvents& E, const IntervalRoute& R, uint32_t n,
                  cudaStream_t s, uint32_t* kernels) {
  int rc;
  uint32_t k = 0;
  if (!R.lo.empty()) {
    RunPlan P;
    if ((rc = plan_intervals(c, R.lo.data(), R.hi.data(), (uint32_t)R.lo.size(), 0, &P))) return rc;
    SieveArgs a;
    if ((rc = launch_plan_ws(c, W, E, P, false, 0, false, s, 0, &a))) return rc;
    k = (uint32_t)(&W == &c->ws ? c->last_kernels : 3) + 1;
    const bool identity = R.lo.size() == n;
    if (!identity) {
      if ((rc = W.sh_map.ensure(sizeof(uint32_t) * R.map.size()))) return rc;
      CUDA_TRY(cudaMemcpyAsync(W.sh_map.p, R.map.data(), sizeof(uint32_t) * R.map.size(), cudaMemcpyHostToDevice, s));
    }
    if (launch_interval_finalize(a, W.out.as<IntervalOut>(), W.istats.as<voss_interval_stats>(),
                                 identity ? nullptr : W.sh_map.as<uint32_t>(), s))
      return fail(VOSS_ERR_CUDA, "interval finalize launch failed");
  } else {
    // no sieve launch: the events bracket the Miller-Rabin path alone
    if ((rc = W.counters.ensure(sizeof(uint32_t) * kCtrWords))) return rc;
    for (cudaEvent_t e : {E.ev0, E.evp, E.ev1})
      if (e) CUDA_TRY(cudaEventRecord(e, s));
    CUDA_TRY(cudaMemsetAsync(W.counters.p, 0, sizeof(uint32_t) * kCtrWords, s));
  }
  if (!R.sv.empty()) {
    NvtxRange r("short intervals by Miller-Rabin");
    const uint64_t nc = R.n_cand;
    if ((rc = W.sh_iv.ensure(sizeof(ShortInterval) * R.sv.size())) || (rc = W.mr_in.ensure(8 * std::max<uint64_t>(nc, 1))) ||
        (rc = W.mr_out.ensure(std::max<uint64_t>(nc, 1))) || (rc = W.mr_work.ensure(sizeof(uint32_t) * (nc + 8))))
      return rc;
    CUDA_TRY(cudaMemcpyAsync(W.sh_iv.p, R.sv.data(), sizeof(ShortInterval) * R.sv.size(), cudaMemcpyHostToDevice, s));
    uint32_t* work = W.mr_work.as<uint32_t>();
    if (launch_short_intervals(W.sh_iv.as<ShortInterval>(), (uint32_t)R.sv.size(), nc, W.mr_in.as<uint64_t>(),
                               W.mr_out.as<uint8_t>(), work + 8, work, W.istats.as<voss_interval_stats>(), c->sm_count,
                               s))
      return fail(VOSS_ERR_CUDA, "short-interval launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    k += nc ? 4 : 1;
  }
  if (E.ev2) CUDA_TRY(cudaEventRecord(E.ev2, s));  // finalize and the Miller-Rabin path count in the launch's time
  if (kernels) *kernels = k;
  return VOSS_OK;
}

int check_device_error(const uint32_t* ctr_host) {
  if (ctr_host[kCtrError] & kErrBounds) return fail(VOSS_ERR_DEVICE, "kernel bounds check failed");
  if (ctr_host[kCtrError] & kErrOverflowList) return fail(VOSS_ERR_DEVICE, "gap overflow list full");
  if (ctr_host[kCtrError]) return fail(VOSS_ERR_DEVICE, "kernel error word 0x%x", ctr_host[kCtrError]);
  return VOSS_OK;
}

// Small primes 2, 3, 5 are outside the wheel; return those in [lo, hi).
std::vector<uint64_t> small_primes_in(uint64_t lo, uint64_t hi) {
  std::vector<uint64_t> v;
  for (uint64_t p : {2ull, 3ull, 5ull})
    if (p >= lo && p < hi) v.push_back(p);
  return v;
}

void add_small_primes(voss_interval_stats& st, uint64_t lo, uint64_t hi) {
  st.lo = lo;
  st.hi = hi;
  const std::vector<uint64_t> sp = small_primes_in(lo, hi);
  if (sp.empty()) return;
  std::vector<uint64_t> seq = sp;
  if (st.first_prime) seq.push_back(st.first_prime);
  uint64_t sm_max = 0, sm_lo = 0;
  for (size_t k = 1; k < seq.size(); ++k) {
    const uint64_t g = seq[k] - seq[k - 1];
    st.gap_hist[g >> 1]++;
    if (g > sm_max) {
      sm_max = g;
      sm_lo = seq[k - 1];
    }
  }
  if (sm_max >= st.max_gap) {  // earlier pairs win ties
    st.max_gap = sm_max;
    st.max_gap_lo = sm_lo;
  }
  st.prime_count += sp.size();
  if (!st.last_prime) st.last_prime = sp.back();
  st.first_prime = sp.front();
}

int row30(uint64_t p) {
  const int r = (int)(p % 30);
  for (int i = 0; i < 8; ++i)
    if (kW30[i] == r) return i;
  return -1;
}

// Fold the device accumulators of one range into voss_range_stats (without large gaps).
void finalize_range(const unsigned long long* acc, const IntervalOut& o, uint64_t lo, uint64_t hi,
                    uint32_t flags, uint64_t seg_num, const std::vector<OverflowGap>& over,
                    voss_range_stats* st) {
  const bool compat = (flags & VOSS_FLAG_REF_COMPAT) != 0;
  std::memset(st, 0, sizeof(*st));
  st->lo = lo;
  st->hi = hi;
  st->flags = flags;
  st->seg_num = compat ? seg_num : 0;
  st->prime_count = acc[kAccCount];
  // gap histogram: bins g/2; for g < 100 add the per-residue bins
  for (int b = 1; b < kHistBins; ++b) {
    uint64_t v = acc[kAccHist + b];
    if (b < kModqBins)
      for (int r = 0; r < 8; ++r) v += acc[kAccModq + r * kModqBins + b];
    if (2 * b < VOSS_MAX_GAP) st->gap_hist[2 * b] += v;
  }
  for (const OverflowGap& g : over)
    if (g.gap < VOSS_MAX_GAP) st->gap_hist[g.gap]++;
  // per-residue gap histogram rows (q = 6 rows {1,5}, then q = 30 rows W30)
  for (int r = 0; r < 8; ++r) {
    const int row6 = (kW30[r] % 6 == 1) ? 0 : 1;
    for (int b = 1; b < kModqBins; ++b) {
      const uint64_t v = acc[kAccModq + r * kModqBins + b];
      st->modq_gap[row6][2 * b] += v;
      st->modq_gap[2 + r][2 * b] += v;
    }
  }
  // residue classes -> mod 4 and mod q (840 = 0 mod 3,4,5,6,7,8,12,30; 4290 = 0 mod 11,13)
  int off[VOSS_NUM_Q];
  for (int qi = 0, s = 0; qi < VOSS_NUM_Q; ++qi) {
    off[qi] = s;
    s += kQ[qi];
  }
  for (int c = 0; c < 28; ++c)
    for (int r = 0; r < 8; ++r) {
      const uint64_t n = acc[kAccCls28 + c * 8 + r];
      if (!n) continue;
      const uint64_t v = 30ull * c + kW30[r];
      if ((v & 3) == 1) st->mod4[0] += n;
      else if ((v & 3) == 3) st->mod4[1] += n;
      for (int qi = 0; qi < VOSS_NUM_Q; ++qi) {
        const int q = kQ[qi];
        if (q == 11 || q == 13) continue;
        st->modq[off[qi] + (int)(v % q)] += n;
      }
    }
  for (int c = 0; c < 143; ++c)
    for (int r = 0; r < 8; ++r) {
      const uint64_t n = acc[kAccCls143 + c * 8 + r];
      if (!n) continue;
      const uint64_t v = 30ull * c + kW30[r];
      st->modq[off[6] + (int)(v % 11)] += n;
      st->modq[off[8] + (int)(v % 13)] += n;
    }
  st->first_prime = o.first;
  st->last_prime = o.last;
  st->max_gap = o.max_gap;
  st->max_gap_lo = o.max_gap_lo;

  // primes 2, 3, 5 and their gaps (they come first in the order of primes)
  const std::vector<uint64_t> sp = small_primes_in(lo, hi);
  if (!sp.empty()) {
    std::vector<uint64_t> seq = sp;
    if (o.first) seq.push_back(o.first);
    uint64_t sm_max = 0, sm_lo = 0;
    for (size_t i = 1; i < seq.size(); ++i) {
      const uint64_t g = seq[i] - seq[i - 1];
      if (g < VOSS_MAX_GAP) st->gap_hist[g]++;
      if (g > sm_max) {
        sm_max = g;
        sm_lo = seq[i - 1];
      }
    }
    if (sm_max >= st->max_gap) {  // earlier pairs win ties
      st->max_gap = sm_max;
      st->max_gap_lo = sm_lo;
    }
    st->prime_count += sp.size();
    st->first_prime = sp.front();
    if (!o.last) st->last_prime = sp.back();
    for (uint64_t p : sp) {
      if ((p & 3) == 1) st->mod4[0]++;
      else if ((p & 3) == 3) st->mod4[1]++;
      if (!compat)
        for (int qi = 0; qi < VOSS_NUM_Q; ++qi) st->modq[off[qi] + (int)(p % kQ[qi])]++;
    }
  }
}

int fetch_common(voss_ctx* c, uint32_t n_iv, std::vector<unsigned long long>& acc,
                 std::vector<IntervalOut>& outs, uint32_t* ctr, std::vector<OverflowGap>& over,
                 bool want_acc) {
  NvtxRange r("fetch statistics");
  cudaStream_t s = c->stream;
  CUDA_TRY(cudaMemcpyAsync(ctr, c->ws.counters.p, sizeof(uint32_t) * kCtrWords, cudaMemcpyDeviceToHost, s));
  outs.resize(std::max<uint32_t>(1, n_iv));
  CUDA_TRY(cudaMemcpyAsync(outs.data(), c->ws.out.p, sizeof(IntervalOut) * n_iv, cudaMemcpyDeviceToHost, s));
  if (want_acc) {
    acc.resize((size_t)kAccStride * std::max<uint32_t>(1, n_iv));
    CUDA_TRY(cudaMemcpyAsync(acc.data(), c->ws.acc.p, sizeof(unsigned long long) * kAccStride * n_iv,
                             cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  int rc = check_device_error(ctr);
  if (rc) return rc;
  const uint32_t no = std::min(ctr[kCtrOver], kOverCap);
  over.resize(no);
  if (no) CUDA_TRY(cudaMemcpy(over.data(), c->ws.over.p, sizeof(OverflowGap) * no, cudaMemcpyDeviceToHost));
  return VOSS_OK;
}

int run_range_device(voss_ctx* c, uint64_t lo, uint64_t hi, uint32_t flags, uint64_t seg_num,
                     uint64_t large_cap, cudaStream_t s) {
  const bool compat = (flags & VOSS_FLAG_REF_COMPAT) != 0;
  if (hi < lo) return fail(VOSS_ERR_ARG, "hi < lo");
  if (hi > c->max_hi) return fail(VOSS_ERR_RANGE, "hi = %" PRIu64 " exceeds the context limit %" PRIu64, hi, c->max_hi);
  uint64_t seg_k = 0;
  if (compat) {
    if (seg_num == 0 || seg_num % 30) return fail(VOSS_ERR_ARG, "seg_num must be a positive multiple of 30");
    seg_k = seg_num / 30;
    const uint64_t tile_bytes = 4ull * c->tune.block_threads * c->tune.chunk_words;
    if (seg_k < tile_bytes)
      return fail(VOSS_ERR_ARG, "seg_num/30 = %" PRIu64 " is below the tile size %" PRIu64 " bytes", seg_k, tile_bytes);
  }
  RunPlan P;
  int rc;
  {
    NvtxRange r("plan");
    rc = plan_intervals(c, &lo, &hi, 1, seg_k, &P);
  }
  if (rc) return rc;
  {
    NvtxRange r("launch");
    rc = launch_plan(c, P, true, large_cap, false, s);
  }
  if (rc) return rc;
  c->have_range = true;
  c->r_lo = lo;
  c->r_hi = hi;
  c->r_seg = compat ? seg_num : 0;
  c->r_flags = flags;
  c->r_tiles = P.n_tiles;
  c->r_large_cap = std::min(std::max(large_cap, (uint64_t)1), kMaxLargeCap);
  return VOSS_OK;
}

// The first n device large-gap records, sorted by position on the device (positions < hi), in
// the context's pinned staging.
int stage_large_sorted(voss_ctx* c, uint64_t n, uint64_t hi, voss_large_gap** out) {
  if (n > c->h_large_cap) {
    if (c->h_large) cudaFreeHost(c->h_large);
    c->h_large = nullptr;
    c->h_large_cap = 0;
    const size_t cap = (size_t)n + n / 4 + 1024;
    if (cudaMallocHost(&c->h_large, cap * sizeof(voss_large_gap)) != cudaSuccess) {
      c->h_large = nullptr;
      return fail(VOSS_ERR_NOMEM, "cudaMallocHost of the large-gap staging failed");
    }
    c->h_large_cap = cap;
  }
  *out = c->h_large;
  if (n == 0) return VOSS_OK;
  NvtxRange r("sort and copy large gaps");
  Workspace& W = c->ws;
  cudaStream_t s = c->stream;
  const int end_bit = hi > 1 ? 64 - __builtin_clzll(hi - 1) : 1;  // bits in which positions can differ
  const size_t tb = large_sort_temp_bytes((uint32_t)n, end_bit);
  int rc;
  if ((rc = W.ls_keys.ensure(16 * n)) || (rc = W.ls_idx.ensure(8 * n)) || (rc = W.ls_temp.ensure(std::max<size_t>(tb, 1))) ||
      (rc = W.ls_sorted.ensure(sizeof(voss_large_gap) * n)))
    return rc;
  if (launch_large_sort(W.large.as<LargeGapDev>(), (uint32_t)n, end_bit, W.ls_keys.as<unsigned long long>(),
                        W.ls_idx.as<uint32_t>(), W.ls_temp.p, tb, W.ls_sorted.as<LargeGapDev>(), c->sm_count, s))
    return fail(VOSS_ERR_CUDA, "large-gap sort failed: %s", cudaGetErrorString(cudaGetLastError()));
  CUDA_TRY(cudaMemcpyAsync(c->h_large, W.ls_sorted.p, sizeof(voss_large_gap) * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return VOSS_OK;
}

int fetch_range(voss_ctx* c, voss_range_stats* st, voss_large_gap* large, uint64_t large_cap,
                uint64_t* written) {
  if (!c->have_range) return fail(VOSS_ERR_STATE, "no range has been sieved on this context");
  std::vector<unsigned long long> acc;
  std::vector<IntervalOut> outs;
  std::vector<OverflowGap> over;
  uint32_t ctr[kCtrWords];
  int rc = fetch_common(c, 1, acc, outs, ctr, over, true);
  if (rc) return rc;
  cudaEventElapsedTime(&c->sieve_ms, c->ev0, c->ev1);
  cudaEventElapsedTime(&c->total_ms, c->ev0, c->ev2);
  {
    NvtxRange r("finalize statistics");
    finalize_range(acc.data(), outs[0], c->r_lo, c->r_hi, c->r_flags, c->r_seg, over, st);
  }
  const uint64_t found = ctr[kCtrLarge];
  st->large_total = found;
  const uint64_t ondev = std::min<uint64_t>(found, c->r_large_cap);
  const uint64_t w = std::min<uint64_t>(ondev, large ? large_cap : 0);
  if (w) {
    voss_large_gap* lg = nullptr;
    if ((rc = stage_large_sorted(c, ondev, c->r_hi, &lg))) return rc;
    std::memcpy(large, lg, sizeof(voss_large_gap) * w);
  }
  if (written) *written = w;
  return VOSS_OK;
}

}  // namespace

// =====================================================================================
// C ABI
// =====================================================================================
using namespace voss_host;

extern "C" {

VOSS_API const char* voss_version(void) { return "voss-b200 0.1 (sm_100a)"; }

VOSS_API const char* voss_last_error(void) { return g_err.c_str(); }

VOSS_API int voss_device_count(int* count) {
  if (!count) return fail(VOSS_ERR_ARG, "count is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) n = 0;
  *count = n;
  return VOSS_OK;
}

VOSS_API int voss_ctx_create(int device, uint64_t max_hi, voss_ctx** out) {
  if (!out) return fail(VOSS_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (max_hi < 8 || max_hi > kMaxHi) return fail(VOSS_ERR_ARG, "max_hi must be in [8, 2^62]");
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(VOSS_ERR_NODEV, "no CUDA device");
  if (device < 0 || device >= n) return fail(VOSS_ERR_ARG, "device %d out of range", device);
  voss_ctx* c = new voss_ctx();
  c->device = device;
  c->max_hi = max_hi;
  auto bail = [&](int code) {
    voss_ctx_destroy(c);
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) return bail(fail(VOSS_ERR_CUDA, "cudaSetDevice failed"));
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail(fail(VOSS_ERR_CUDA, "cudaGetDeviceProperties failed"));
  c->sm_count = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_copy, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_stage[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->ev_stage[1], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
      cudaEventCreate(&c->ev2) != cudaSuccess || cudaEventCreate(&c->evp) != cudaSuccess)
    return bail(fail(VOSS_ERR_CUDA, "stream/event creation failed"));
  c->primes = base_primes(isqrt_u64(max_hi - 1));
  const size_t np = std::max<size_t>(1, c->primes.size());
  int rc;
  if ((rc = c->d_primes.ensure(np * sizeof(uint32_t))) || (rc = c->d_magic.ensure(np * sizeof(uint64_t))) ||
      (rc = c->d_pretab.ensure(kPreWords * sizeof(uint32_t))))
    return bail(rc);
  std::vector<uint64_t> magic(np, 0);
  for (size_t i = 0; i < c->primes.size(); ++i) magic[i] = ~0ull / c->primes[i];
  std::vector<uint32_t> pre(kPreWords);
  build_presieve_tables(pre.data());
  if (!c->primes.empty()) {
    if (cudaMemcpy(c->d_primes.p, c->primes.data(), c->primes.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(c->d_magic.p, magic.data(), c->primes.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(VOSS_ERR_CUDA, "base prime upload failed"));
  }
  if (cudaMemcpy(c->d_pretab.p, pre.data(), kPreWords * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(VOSS_ERR_CUDA, "presieve table upload failed"));
  voss_tuning t{};
  if ((rc = apply_tuning(c, t))) return bail(rc);
  if (const char* lim = std::getenv("VOSS_STAGE_LIMIT")) {
    const unsigned long long v = std::strtoull(lim, nullptr, 10);
    if (v) c->stage_limit = std::max<size_t>(1024, (size_t)v);
  }
  *out = c;
  return VOSS_OK;
}

VOSS_API void voss_ctx_destroy(voss_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev2) cudaEventDestroy(c->ev2);
  if (c->evp) cudaEventDestroy(c->evp);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->ev_copy) cudaEventDestroy(c->ev_copy);
  if (c->h_large) cudaFreeHost(c->h_large);
  for (int b = 0; b < 2; ++b) {
    if (c->h_stage[b]) cudaFreeHost(c->h_stage[b]);
    if (c->ev_stage[b]) cudaEventDestroy(c->ev_stage[b]);
  }
  delete c;
}

VOSS_API int voss_ctx_info(const voss_ctx* c, uint64_t* max_hi, uint64_t* n_base_primes, int* sm_count) {
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  if (max_hi) *max_hi = c->max_hi;
  if (n_base_primes) {
    // base primes >= 7 up to isqrt(max_hi - 1): the table (>= 37) plus 7..31 when in range
    const uint64_t lim = isqrt_u64(c->max_hi - 1);
    uint64_t small = 0;
    for (uint64_t p : {7ull, 11ull, 13ull, 17ull, 19ull, 23ull, 29ull, 31ull})
      if (p <= lim) ++small;
    *n_base_primes = c->primes.size() + small;
  }
  if (sm_count) *sm_count = c->sm_count;
  return VOSS_OK;
}

VOSS_API int voss_ctx_set_tuning(voss_ctx* c, const voss_tuning* t) {
  if (!c || !t) return fail(VOSS_ERR_ARG, "NULL argument");
  return apply_tuning(c, *t);
}

VOSS_API int voss_ctx_get_tuning(const voss_ctx* c, voss_tuning* t) {
  if (!c || !t) return fail(VOSS_ERR_ARG, "NULL argument");
  *t = c->tune;
  return VOSS_OK;
}

VOSS_API int voss_sieve_range_device(voss_ctx* c, uint64_t lo, uint64_t hi, uint32_t flags,
                                     uint64_t seg_num, void* stream) {
  NvtxRange nvtx_("voss_sieve_range_device");
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  cudaSetDevice(c->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int rc = run_range_device(c, lo, hi, flags, seg_num, kDefaultLargeCap, s);
  if (rc) return rc;
  if (s != c->stream) {  // later fetches run on the context stream
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(e, s));
    CUDA_TRY(cudaStreamWaitEvent(c->stream, e, 0));
    cudaEventDestroy(e);
  }
  return VOSS_OK;
}

VOSS_API int voss_fetch_range(voss_ctx* c, voss_range_stats* st, voss_large_gap* large,
                              uint64_t large_cap, uint64_t* written) {
  NvtxRange nvtx_("voss_fetch_range");
  if (!c || !st) return fail(VOSS_ERR_ARG, "NULL argument");
  cudaSetDevice(c->device);
  return fetch_range(c, st, large, large_cap, written);
}

VOSS_API int voss_sieve_range(voss_ctx* c, uint64_t lo, uint64_t hi, uint32_t flags, uint64_t seg_num,
                              voss_range_stats* st, voss_large_gap* large, uint64_t large_cap,
                              uint64_t* written) {
  NvtxRange nvtx_("voss_sieve_range");
  if (!c || !st) return fail(VOSS_ERR_ARG, "NULL argument");
  cudaSetDevice(c->device);
  int rc = run_range_device(c, lo, hi, flags, seg_num, std::max(large_cap, kDefaultLargeCap), c->stream);
  if (rc) return rc;
  return fetch_range(c, st, large, large_cap, written);
}

VOSS_API int voss_last_kernel_ms(const voss_ctx* c, double* sieve_ms, double* total_ms) {
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  cudaSetDevice(c->device);
  float a = 0, b = 0;
  CUDA_TRY(cudaEventSynchronize(c->ev2));
  CUDA_TRY(cudaEventElapsedTime(&a, c->ev0, c->ev1));
  CUDA_TRY(cudaEventElapsedTime(&b, c->ev0, c->ev2));
  if (sieve_ms) *sieve_ms = a;
  if (total_ms) *total_ms = b;
  return VOSS_OK;
}

VOSS_API int voss_last_phase_ms(const voss_ctx* c, double* prepass_ms, double* tile_ms, double* tail_ms,
                                uint32_t* kernels) {
  NvtxRange nvtx_("voss_last_phase_ms");
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  cudaSetDevice(c->device);
  float a = 0, b = 0, t = 0;
  CUDA_TRY(cudaEventSynchronize(c->ev2));
  CUDA_TRY(cudaEventElapsedTime(&a, c->ev0, c->evp));
  CUDA_TRY(cudaEventElapsedTime(&b, c->evp, c->ev1));
  CUDA_TRY(cudaEventElapsedTime(&t, c->ev1, c->ev2));
  if (prepass_ms) *prepass_ms = a;
  if (tile_ms) *tile_ms = b;
  if (tail_ms) *tail_ms = t;
  if (kernels) *kernels = c->last_kernels;
  return VOSS_OK;
}

VOSS_API int voss_sieve_intervals(voss_ctx* c, const uint64_t* lo, const uint64_t* hi, uint32_t n,
                                  voss_interval_stats* out) {
  NvtxRange nvtx_("voss_sieve_intervals");
  if (!c || (n && (!lo || !hi || !out))) return fail(VOSS_ERR_ARG, "NULL argument");
  cudaSetDevice(c->device);
  for (uint32_t i = 0; i < n; ++i) {
    if (hi[i] < lo[i]) return fail(VOSS_ERR_ARG, "interval %u has hi < lo", i);
    if (hi[i] > c->max_hi) return fail(VOSS_ERR_RANGE, "interval %u exceeds the context limit", i);
  }
  if (n == 0) return VOSS_OK;
  Workspace& W = c->ws;
  cudaStream_t s = c->stream;
  int rc;
  IntervalRoute R;
  route_intervals(c, lo, hi, n, 1ull << 32, &R);
  LaunchEvents E;
  E.ev0 = c->ev0;
  E.evp = c->evp;
  E.ev1 = c->ev1;
  E.ev2 = c->ev2;
  uint32_t kernels = 0;
  if ((rc = W.istats.ensure(sizeof(voss_interval_stats) * n))) return rc;
  if ((rc = launch_routed(c, W, E, R, n, s, &kernels))) return rc;
  c->last_kernels = kernels;
  uint32_t ctr[kCtrWords];
  CUDA_TRY(cudaMemcpyAsync(ctr, W.counters.p, sizeof(ctr), cudaMemcpyDeviceToHost, s));
  // large results (8 KB per interval) come back through pinned staging, copied out by host threads
  // (two halves over the two buffers: the second crosses while the first is copied out)
  const size_t res_bytes = sizeof(voss_interval_stats) * n;
  const bool staged = res_bytes >= (8u << 20);
  if (staged) {
    if ((rc = ensure_stage(c, (res_bytes + 15) / 16))) return rc;
    if ((rc = stage_out(c, out, W.istats.p, res_bytes, s))) return rc;
  } else {
    CUDA_TRY(cudaMemcpyAsync(out, W.istats.p, res_bytes, cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  if ((rc = check_device_error(ctr))) return rc;
  cudaEventElapsedTime(&c->sieve_ms, c->ev0, c->ev1);
  cudaEventElapsedTime(&c->total_ms, c->ev0, c->ev2);
  for (uint32_t i = 0; i < n; ++i) add_small_primes(out[i], lo[i], hi[i]);
  return VOSS_OK;
}

VOSS_API int voss_gaps_at_least(voss_ctx* c, uint64_t lo, uint64_t hi, uint32_t min_gap, voss_large_gap* out,
                                uint64_t cap, uint64_t* count) {
  NvtxRange nvtx_("voss_gaps_at_least");
  if (!c || !count || (cap && !out)) return fail(VOSS_ERR_ARG, "NULL argument");
  if (min_gap < 3) return fail(VOSS_ERR_ARG, "min_gap must be at least 3");
  if (hi < lo) return fail(VOSS_ERR_ARG, "hi < lo");
  if (hi > c->max_hi) return fail(VOSS_ERR_RANGE, "hi exceeds the context limit");
  cudaSetDevice(c->device);
  RunPlan P;
  int rc = plan_intervals(c, &lo, &hi, 1, 0, &P);
  if (rc) return rc;
  const uint64_t devcap = std::min<uint64_t>(std::max<uint64_t>(cap, 1), kMaxLargeCap);
  rc = launch_plan(c, P, true, devcap, false, c->stream, min_gap);
  if (rc) return rc;
  uint32_t ctr[kCtrWords];
  CUDA_TRY(cudaMemcpyAsync(ctr, c->ws.counters.p, sizeof(ctr), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if ((rc = check_device_error(ctr))) return rc;
  const uint64_t found = ctr[kCtrLarge];
  *count = found;
  const uint64_t w = std::min<uint64_t>(std::min<uint64_t>(found, devcap), cap);
  if (w) {
    voss_large_gap* v = nullptr;
    if ((rc = stage_large_sorted(c, std::min<uint64_t>(found, devcap), hi, &v))) return rc;
    std::memcpy(out, v, sizeof(voss_large_gap) * w);
  }
  return VOSS_OK;
}

VOSS_API int voss_primes_range(voss_ctx* c, uint64_t lo, uint64_t hi, uint64_t* out, uint64_t cap,
                               uint64_t* count) {
  NvtxRange nvtx_("voss_primes_range");
  if (!c || !count || (cap && !out)) return fail(VOSS_ERR_ARG, "NULL argument");
  if (hi < lo) return fail(VOSS_ERR_ARG, "hi < lo");
  if (hi > c->max_hi) return fail(VOSS_ERR_RANGE, "hi exceeds the context limit");
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  RunPlan P;
  int rc = plan_intervals(c, &lo, &hi, 1, 0, &P);
  if (rc) return rc;
  // pass 1: per-tile counts
  rc = launch_plan(c, P, false, 0, false, s);
  if (rc) return rc;
  std::vector<TilePartial> parts(P.n_tiles);
  if (P.n_tiles)
    CUDA_TRY(cudaMemcpyAsync(parts.data(), c->ws.partials.p, sizeof(TilePartial) * P.n_tiles, cudaMemcpyDeviceToHost, s));
  uint32_t ctr[kCtrWords];
  CUDA_TRY(cudaMemcpyAsync(ctr, c->ws.counters.p, sizeof(ctr), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if ((rc = check_device_error(ctr))) return rc;
  std::vector<unsigned long long> offs(std::max<uint32_t>(1, P.n_tiles));
  uint64_t total = 0;
  for (uint32_t t = 0; t < P.n_tiles; ++t) {
    offs[t] = total;
    total += parts[t].count;
  }
  const std::vector<uint64_t> sp = small_primes_in(lo, hi);
  *count = total + sp.size();
  uint64_t k = 0;
  for (uint64_t p : sp) {
    if (k < cap) out[k] = p;
    ++k;
  }
  if (total == 0 || k >= cap) return VOSS_OK;
  const uint64_t room = std::min<uint64_t>(total, cap - k);
  if ((rc = c->ws.offsets.ensure(sizeof(unsigned long long) * offs.size()))) return rc;
  if ((rc = c->ws.emit.ensure(sizeof(unsigned long long) * room))) return rc;
  CUDA_TRY(cudaMemcpyAsync(c->ws.offsets.p, offs.data(), sizeof(unsigned long long) * P.n_tiles, cudaMemcpyHostToDevice, s));
  // pass 2: write (out_cap is the buffer size, which may exceed `room`)
  rc = launch_plan(c, P, false, 0, true, s);
  if (rc) return rc;
  CUDA_TRY(cudaMemcpyAsync(out + k, c->ws.emit.p, sizeof(uint64_t) * room, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(ctr, c->ws.counters.p, sizeof(ctr), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return check_device_error(ctr);
}

VOSS_API int voss_mr_verify_device(voss_ctx* c, const uint64_t* d_n, uint64_t count, uint8_t* d_out,
                                   void* stream) {
  NvtxRange nvtx_("voss_mr_verify_device");
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  if (count && (!d_n || !d_out)) return fail(VOSS_ERR_ARG, "NULL argument");
  if (count > 0xFFFFFFFFull) return fail(VOSS_ERR_ARG, "count must be < 2^32 per call");
  cudaSetDevice(c->device);
  cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
  int rc;
  if ((rc = c->ws.mr_work.ensure(sizeof(uint32_t) * (std::max<uint64_t>(count, 1) + 8)))) return rc;
  uint32_t* work = c->ws.mr_work.as<uint32_t>();
  if (launch_mr(d_n, count, d_out, work + 8, work, s, c->sm_count))
    return fail(VOSS_ERR_CUDA, "Miller-Rabin launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return VOSS_OK;
}

VOSS_API int voss_mr_verify(voss_ctx* c, const uint64_t* n, uint64_t count, uint8_t* is_prime) {
  NvtxRange nvtx_("voss_mr_verify");
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  if (count == 0) return VOSS_OK;
  if (!n || !is_prime) return fail(VOSS_ERR_ARG, "NULL argument");
  if (count > 0xFFFFFFFFull) return fail(VOSS_ERR_ARG, "count must be < 2^32 per call");
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  Workspace& W = c->ws;
  int rc;
  // context-owned, grow-only buffers: repeated calls do not allocate.  The candidates cross in
  // chunks on the copy stream while the previous chunk is tested on `stream`.  Large batches go
  // through two pinned staging buffers that host threads fill (chunk i + 1 is copied in while
  // chunk i crosses and chunk i - 1 is tested), and the verdicts come back the same way; small
  // ones are copied straight from the caller's memory.
  const bool staged = count >= (1ull << 20);
  if (staged && (rc = ensure_stage(c, std::min<uint64_t>(count, 1ull << 24)))) return rc;
  const uint64_t kChunk = staged ? c->h_stage_cap : (1ull << 24);  // candidates per launch
  const uint64_t per = std::min(count, kChunk);
  if ((rc = W.mr_in.ensure(count * 8)) || (rc = W.mr_out.ensure(count)) ||
      (rc = W.mr_work.ensure(sizeof(uint32_t) * (per + 8))))
    return rc;
  uint64_t* d_in = W.mr_in.as<uint64_t>();
  uint8_t* d_out = W.mr_out.as<uint8_t>();
  uint32_t* work = W.mr_work.as<uint32_t>();
  uint64_t i = 0;
  for (uint64_t off = 0; off < count; off += kChunk, ++i) {
    const uint64_t k = std::min(kChunk, count - off);
    if (staged) {
      const int b = (int)(i & 1);
      CUDA_TRY(cudaEventSynchronize(c->ev_stage[b]));  // buffer b's previous transfer is done
      parallel_copy(c->h_stage[b], n + off, k * 8);
      CUDA_TRY(cudaMemcpyAsync(d_in + off, c->h_stage[b], k * 8, cudaMemcpyHostToDevice, c->copy_stream));
      CUDA_TRY(cudaEventRecord(c->ev_stage[b], c->copy_stream));
    } else {
      CUDA_TRY(cudaMemcpyAsync(d_in + off, n + off, k * 8, cudaMemcpyHostToDevice, c->copy_stream));
    }
    CUDA_TRY(cudaEventRecord(c->ev_copy, c->copy_stream));
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_copy, 0));
    if (launch_mr(d_in + off, k, d_out + off, work + 8, work, s, c->sm_count))
      return fail(VOSS_ERR_CUDA, "Miller-Rabin launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  if (!staged) {
    CUDA_TRY(cudaMemcpyAsync(is_prime, d_out, count, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaStreamSynchronize(s));
    return VOSS_OK;
  }
  // verdicts: chunk j crosses into buffer j & 1 while chunk j - 1 is copied out by host threads
  // (the input transfers are complete: every launch on `stream` waited for them)
  if ((rc = stage_out(c, is_prime, d_out, count, s))) return rc;
  CUDA_TRY(cudaStreamSynchronize(s));
  return VOSS_OK;
}

VOSS_API int voss_prove_gaps(voss_ctx* c, const uint64_t* p_after, const int32_t* gap, uint64_t count,
                             uint8_t* ok) {
  NvtxRange nvtx_("voss_prove_gaps");
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  if (count == 0) return VOSS_OK;
  if (!p_after || !gap || !ok) return fail(VOSS_ERR_ARG, "NULL argument");
  if (count > 0x7FFFFFFFull) return fail(VOSS_ERR_ARG, "count must be < 2^31 per call");
  cudaSetDevice(c->device);
  cudaStream_t s = c->stream;
  Workspace& W = c->ws;  // context-owned, grow-only buffers: repeated calls do not allocate
  int rc;
  if ((rc = W.pg_pa.ensure(count * 8)) || (rc = W.pg_gap.ensure(count * 4)) || (rc = W.pg_ok.ensure(count)) ||
      (rc = W.mr_in.ensure(2 * count * 8)) || (rc = W.mr_out.ensure(2 * count)) ||
      (rc = W.mr_work.ensure(sizeof(uint32_t) * (2 * count + 8))))
    return rc;
  // large batches cross through the pinned staging buffers (filled and emptied by host threads)
  const bool staged = count >= (1ull << 20);
  if (staged) {
    if ((rc = ensure_stage(c, (count + 1) / 2)) || (rc = stage_in(c, W.pg_pa.p, p_after, count * 8, s)) ||
        (rc = stage_in(c, W.pg_gap.p, gap, count * 4, s)))
      return rc;
  } else {
    CUDA_TRY(cudaMemcpyAsync(W.pg_pa.p, p_after, count * 8, cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(W.pg_gap.p, gap, count * 4, cudaMemcpyHostToDevice, s));
  }
  uint32_t* work = W.mr_work.as<uint32_t>();
  if (launch_prove_gaps(W.pg_pa.as<uint64_t>(), W.pg_gap.as<int32_t>(), count, W.pg_ok.as<uint8_t>(),
                        W.mr_in.as<uint64_t>(), W.mr_out.as<uint8_t>(), work + 8, work, s, c->sm_count))
    return fail(VOSS_ERR_CUDA, "gap proof launch failed");
  if (staged) {
    if ((rc = stage_out(c, ok, W.pg_ok.p, count, s))) return rc;
  } else {
    CUDA_TRY(cudaMemcpyAsync(ok, W.pg_ok.p, count, cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  return VOSS_OK;
}

VOSS_API int voss_probe_smem_rmw(voss_ctx* c, double* gbs) {
  if (!c || !gbs) return fail(VOSS_ERR_ARG, "NULL argument");
  cudaSetDevice(c->device);
  float ms = 0;
  double bytes = 0;
  if (probe_smem_rmw(c->sm_count, c->stream, &ms, &bytes)) return fail(VOSS_ERR_CUDA, "probe failed");
  *gbs = bytes / (ms * 1e-3) / 1e9;
  return VOSS_OK;
}

VOSS_API int voss_probe_mulmod(voss_ctx* c, double* full_per_s, double* small_per_s) {
  if (!c || !full_per_s || !small_per_s) return fail(VOSS_ERR_ARG, "NULL argument");
  cudaSetDevice(c->device);
  if (probe_mulmod(c->sm_count, c->stream, full_per_s, small_per_s)) return fail(VOSS_ERR_CUDA, "probe failed");
  return VOSS_OK;
}

}  // extern "C"

#ifdef VOSS_PHASE_TIMING
namespace voss {
int read_phase_cycles(unsigned long long* out, int n, bool reset);
}
// Instrumented build only (libvoss_timing.so): cycles per kernel phase summed over CTAs.
extern "C" VOSS_API int voss_debug_phase_cycles(unsigned long long* out, int n, int reset) {
  return voss::read_phase_cycles(out, n, reset != 0) ? VOSS_ERR_CUDA : VOSS_OK;
}
#endif

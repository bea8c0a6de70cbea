// voss_host.h — host-runtime types shared by the C ABI (voss_api.cpp) and the request server
// (voss_server.cpp).  Not installed; the public interface is include/voss.h.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <vector>

#include "voss.h"
#include "voss_internal.h"

namespace voss_host {

// Record a message for voss_last_error() and return `code`.
int fail(int code, const char* fmt, ...);

// NVTX range in the "voss" domain for the lifetime of the object: every API call and its host
// stages (plan, launch, sort, copy) show as named spans on an Nsight Systems timeline.  NVTX 3
// is header-only; with no tool attached a push/pop is a test of one pointer.
inline nvtxDomainHandle_t nvtx_domain() {
  static nvtxDomainHandle_t d = nvtxDomainCreateA("voss");
  return d;
}
struct NvtxRange {
  explicit NvtxRange(const char* name) {
    nvtxEventAttributes_t a = {};
    a.version = NVTX_VERSION;
    a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
    a.messageType = NVTX_MESSAGE_TYPE_ASCII;
    a.message.ascii = name;
    nvtxDomainRangePushEx(nvtx_domain(), &a);
  }
  ~NvtxRange() { nvtxDomainRangePop(nvtx_domain()); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

#define CUDA_TRY(call)                                                                      \
  do {                                                                                      \
    cudaError_t e__ = (call);                                                               \
    if (e__ != cudaSuccess)                                                                 \
      return ::voss_host::fail(VOSS_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e__)); \
  } while (0)

// A grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  int ensure(size_t need);
  template <class T>
  T* as() const {
    return static_cast<T*>(p);
  }
};

// Device memory of one launch of the tile kernel (and of Miller-Rabin batches).
struct Workspace {
  DevBuf iv, partials, acc, out, large, large_iv, over, counters, istats, offsets, emit, mr_work, mr_in, mr_out;
  DevBuf gbm, scat;  // large-prime pre-pass: bitmap of the launch and its interval descriptors
  DevBuf tile_iv;    // interval of each tile, for launches of more than one interval
  DevBuf pg_pa, pg_gap, pg_ok;  // gap proofs: inputs and verdicts (endpoints use mr_in / mr_out / mr_work)
  DevBuf sha_data, sha_off, sha_out;  // certificate hashing: messages, offsets, digests
  DevBuf ls_keys, ls_idx, ls_temp, ls_sorted;  // large-gap list sorted by position (large_sort.cu)
  DevBuf sh_iv, sh_map;  // short intervals by Miller-Rabin (short_iv.cu); sieved intervals' result slots
  // Largest large-prime bitmap this workspace may use; with gbm_fixed the buffers are never
  // grown (server slots size them at creation), and launches that need more skip the pre-pass.
  size_t gbm_budget = 8ull << 30;
  bool gbm_fixed = false;
};

// Events bracketing one launch: ev0 before all of its device work (descriptor copies, memsets),
// ev1 after the tile kernel, ev2 after the stitch/reduce kernels; evp (optional) after the
// large-prime pre-pass, just before the tile kernel.
struct LaunchEvents {
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, evp = nullptr;
};

struct RunPlan {
  std::vector<voss::IntervalDev> iv;
  uint32_t n_tiles = 0;
  uint64_t n_words = 0;
};

enum { kCtrTile = 0, kCtrLarge = 1, kCtrOver = 2, kCtrError = 3, kCtrMrWork = 4, kCtrWords = 8 };

constexpr uint64_t kMaxHi = 1ull << 62;
constexpr uint32_t kOverCap = 1u << 16;
constexpr uint64_t kDefaultLargeCap = 1ull << 22;
// Large-prime pre-pass windows: bitmap bytes per window, inside the 126 MB L2 next to the primes
// the pre-pass reads (23 MB of 32-bit primes below 10^8).  On the 4096-interval batch 48 MB
// windows measured 9.46 ms against 9.62 ms for 32 MB, 9.83 ms for 24 MB and 9.61 ms for 64 MB.
#ifndef VOSS_SCATTER_WINDOW_MB
#define VOSS_SCATTER_WINDOW_MB 48
#endif
constexpr uint64_t kScatterWindowBytes = (uint64_t)VOSS_SCATTER_WINDOW_MB << 20;
constexpr uint64_t kMaxLargeCap = 50000000ull;  // MAX_LARGE_GAPS, src/voss_v7_live.cu:34

}  // namespace voss_host

struct voss_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;  // host-to-device copies overlapped with work on `stream`
  cudaEvent_t ev_copy = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr, evp = nullptr;
  uint64_t max_hi = 0;
  std::vector<uint32_t> primes;  // >= 37
  voss_host::DevBuf d_primes, d_magic, d_pretab;
  voss_tuning tune{};
  int ctas_per_sm = 1;
  voss_host::Workspace ws;
  // last range run
  bool have_range = false;
  uint64_t r_lo = 0, r_hi = 0, r_seg = 0;
  uint32_t r_flags = 0;
  uint32_t r_tiles = 0;
  uint64_t r_large_cap = 0;
  float sieve_ms = 0, total_ms = 0;
  uint32_t last_kernels = 0;  // kernels of the last launch_plan_ws (+ finalize for intervals)
  // host side of the large-gap list: pinned, grow-only staging for the device-to-host copy of
  // the list (sorted on the device), so that repeated calls touch no fresh pages
  voss_large_gap* h_large = nullptr;
  size_t h_large_cap = 0;
  // pinned staging of large host batches (Miller-Rabin candidates in, verdicts out): two
  // buffers, one filled by host threads while the other crosses; ev_stage[b] marks the end of
  // buffer b's last transfer
  uint64_t* h_stage[2] = {nullptr, nullptr};
  size_t h_stage_cap = 0;  // 64-bit entries per buffer
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};
  // most 64-bit entries a staging buffer may hold (larger transfers cross in chunks); the
  // environment variable VOSS_STAGE_LIMIT lowers it when the context is created, so tests can
  // drive the chunked paths with small batches
  size_t stage_limit = ~(size_t)0;
};

namespace voss_host {

// Cut intervals [lo_i, hi_i) into tiles; intervals without wheel integers get no tiles.
int plan_intervals(const voss_ctx* c, const uint64_t* lo, const uint64_t* hi, uint32_t n, uint64_t seg_k,
                   RunPlan* P);
// Queue the tile kernel (+ stitch and reduce unless emit) for plan P on stream s, using the
// workspace W and events E.
int launch_plan_ws(voss_ctx* c, Workspace& W, const LaunchEvents& E, const RunPlan& P, bool want_large,
                   uint64_t large_cap, bool emit, cudaStream_t s, uint32_t min_gap, voss::SieveArgs* args_out);
// A batch of intervals split between the sieve (lo, hi, map = their positions in the batch)
// and the Miller-Rabin path for short intervals at high starts (sv, n_cand candidates).
struct IntervalRoute {
  std::vector<uint64_t> lo, hi;
  std::vector<uint32_t> map;
  std::vector<voss::ShortInterval> sv;
  uint64_t n_cand = 0;
};
// Split [lo_i, hi_i) by the context's mr_route, with at most cand_cap Miller-Rabin candidates.
void route_intervals(const voss_ctx* c, const uint64_t* lo, const uint64_t* hi, uint32_t n, uint64_t cand_cap,
                     IntervalRoute* R);
// Launch a routed batch of n intervals on stream s; all n results land in W.istats (lo, hi and
// the primes 2, 3, 5 are the host's, add_small_primes).  E.ev2 is recorded after the last kernel.
int launch_routed(voss_ctx* c, Workspace& W, const LaunchEvents& E, const IntervalRoute& R, uint32_t n,
                  cudaStream_t s, uint32_t* kernels);
int check_device_error(const uint32_t* ctr_host);
// memcpy split over up to 8 host threads, in parts of at least min_part bytes.
void parallel_copy(void* dst, const void* src, size_t bytes, size_t min_part = 8u << 20);
struct CopySeg {
  const void* src;
  size_t bytes;
};
// The segments copied back to back into dst, split the same way.
void parallel_gather(void* dst, const CopySeg* seg, size_t n_seg, size_t min_part);
std::vector<uint64_t> small_primes_in(uint64_t lo, uint64_t hi);
// Add the primes 2, 3, 5 of [lo, hi) to a device-finalized interval result.
void add_small_primes(voss_interval_stats& st, uint64_t lo, uint64_t hi);

}  // namespace voss_host

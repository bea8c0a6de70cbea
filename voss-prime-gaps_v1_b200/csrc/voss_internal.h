// voss_internal.h — layouts shared by the sm_100a kernels and the C++ host runtime.
//
// Data layout (HBM and shared memory)
//   Wheel-30 bitmap: byte k covers the integers 30k + {1,7,11,13,17,19,23,29}; bit o of the
//   byte is residue W30[o] (the reference's bit index idx = 8k + o, src/voss_v7_live.cu:134-138
//   and :189, read as little-endian 32-bit words).  A tile of the bitmap lives only in shared
//   memory; nothing of it is ever written to HBM.
//   Work queue: intervals [lo, hi) are cut into tiles of `tile_words` 32-bit words; tile t of
//   interval i starts at byte k0_i + 4 * tile_words * (t - tile_begin_i).  Persistent CTAs
//   claim tile indices from one atomic counter.
//   Per-interval accumulators (u64, kAccStride per interval) hold the counters every tile
//   adds into; per-tile partials carry the first/last prime of each tile so that the gaps
//   across tile seams can be added afterwards by the stitch kernel.
#pragma once

#include <cstdint>

namespace voss {

// ---- wheel --------------------------------------------------------------------------
// Packed W30 residues, byte o = W30[o].
constexpr uint64_t kW30Packed = 0x1D1713110D0B0701ull;

// ---- presieve groups (primes applied by word masks, never by clearing loops) ----------
// Group g holds the primes whose product is kPreMod[g]; its table has kPreMod[g] 32-bit
// masks, entry j being the mask of every word W with W = j (mod kPreMod[g]).
constexpr int kPreGroups = 4;
constexpr uint32_t kPreMod[kPreGroups] = {1001u /*7*11*13*/, 323u /*17*19*/, 667u /*23*29*/,
                                          31u /*31*/};
constexpr uint32_t kPreOff[kPreGroups] = {0u, 1001u, 1324u, 1991u};
constexpr uint32_t kPreWords = 2022u;
constexpr uint32_t kFirstSievePrime = 37u;  // the base-prime table starts here

// ---- accumulator layout (u64 words per interval) ----------------------------------------
constexpr int kHistBins = 1024;  // bin g/2 for even gaps g < 2048
constexpr int kModqBins = 50;    // per wheel residue of the lower prime: bin g/2, g < 100
constexpr int kCls28 = 28 * 8;   // (k mod 28, residue index)
constexpr int kCls143 = 143 * 8; // (k mod 143, residue index)
constexpr int kAccCount = 0;
constexpr int kAccHist = 1;
constexpr int kAccHistOver = kAccHist + kHistBins;          // 1025
constexpr int kAccModq = kAccHistOver + 1;                  // 1026
constexpr int kAccCls28 = kAccModq + 8 * kModqBins;         // 1426
constexpr int kAccCls143 = kAccCls28 + kCls28;              // 1650
constexpr int kAccUsed = kAccCls143 + kCls143;              // 2794
constexpr int kAccStride = 2800;

// Shared-memory counter block (u32), same order as the accumulator from kAccHist on, except
// that the class blocks are not wrapped: byte j of a word whose first byte has class c counts
// in class c + j (up to 30 and 145), and the flush adds classes 28..30 / 143..145 to 0..2.
constexpr int kSmCls28Rows = 28 + 3;
constexpr int kSmCls143Rows = 143 + 3;
constexpr int kSmHist = 0;
constexpr int kSmModq = kSmHist + kHistBins;                // 1024
constexpr int kSmCls28 = kSmModq + 8 * kModqBins;           // 1424
constexpr int kSmCls143 = kSmCls28 + 8 * kSmCls28Rows;      // 1672
constexpr int kSmCounters = kSmCls143 + 8 * kSmCls143Rows;  // 2840

constexpr uint32_t kNone = 0xFFFFFFFFu;

// Error word bits raised by kernels.
constexpr uint32_t kErrBounds = 1u;     // a shared/global index failed its check (checked build)
constexpr uint32_t kErrOverflowList = 2u;
constexpr uint32_t kErrInvariant = 4u;

struct IntervalDev {
  uint64_t lo;          // first integer considered by the wheel (>= 7)
  uint64_t hi;          // exclusive
  uint64_t k0;          // first byte of the first tile (multiple of 4)
  uint64_t n_words;     // 32-bit words covering [k0, last byte]
  uint64_t seg_k;       // reference-compat segment length in bytes (0: no segment rule)
  uint64_t gword;       // first word of the interval in the large-prime bitmap (when used)
  uint32_t tile_begin;  // global index of the interval's first tile
  uint32_t n_tiles;
};

// One interval as seen by the large-prime pre-pass (sorted by sqrt_hi, descending).
struct __align__(16) IntervalScatter {
  // vbase = 30 * k0, the integer at bit 0 of the interval's first word.
  // Read for every (prime, interval) pair: 16 B
  double vbase_d;     // vbase rounded to double (for the quotient estimate of vbase mod p)
  uint32_t vbase_lo;  // low 32 bits of vbase (the remainder needs only those, see scatter_large_kernel)
  uint32_t span32;    // min(span, 2^32 - 1)
  // read once per prime (how many intervals it reaches) or when a multiple of p may lie inside
  uint32_t sqrt_hi;   // isqrt(hi - 1), capped to 2^32 - 1
  uint32_t lt32;      // bytes of the interval's bitmap (span / 30) when below 2^31, else 0
  uint64_t span;      // integers covered by the interval's words (120 per word)
  uint64_t gword;     // first word in the large-prime bitmap
  uint64_t vbase;     // for primes >= 2^30 (hi above 2^60)
};

// One interval of the Miller-Rabin path for short intervals (short_iv.cu).
struct ShortInterval {
  uint64_t base;       // 30 * floor(a / 30), a = max(lo, 7)
  uint64_t cand_off;   // its first candidate in the launch's candidate array
  uint32_t j0;         // wheel integers of [base, a)
  uint32_t n_cand;     // wheel integers of [a, hi)
  uint32_t out_index;  // position in the caller's result array
  uint32_t pad;
};

struct TilePartial {
  uint32_t first;    // value offset (from 30 * tile byte 0) of the first prime, kNone if none
  uint32_t last;     // value offset of the last prime
  uint32_t count;
  uint32_t max_gap;  // largest in-tile gap (0 if < 2 primes)
  uint32_t max_lo;   // value offset of its lower prime
  uint32_t bgap;     // gap from the previous non-empty tile's last prime (stitch kernel)
  uint64_t bgap_lo;  // that gap's lower prime
};

struct IntervalOut {
  uint64_t first, last, max_gap, max_gap_lo;
};

struct LargeGapDev {  // same layout as voss_large_gap / the reference's LargeGap
  uint64_t position;
  int32_t gap;
  float merit;
};

struct OverflowGap {
  uint32_t interval;
  uint32_t gap;
};

struct SieveArgs {
  const uint32_t* primes;   // base primes >= 37, ascending
  const uint64_t* magic;    // floor((2^64-1)/p) per prime
  uint32_t n_primes;
  uint32_t p_max;           // the last (largest) base prime, 0 when there is none
  const uint32_t* pretab;   // kPreWords presieve masks
  const IntervalDev* iv;
  const uint32_t* tile_iv;  // interval of each tile (nullptr: found by binary search over iv)
  uint32_t n_intervals;
  uint32_t n_tiles;
  uint32_t tile_words;
  uint32_t chunk_words;     // odd; tile_words = blockDim.x * chunk_words
  uint32_t coop_div;
  uint32_t mult_factor;
  uint32_t walk_sixteenths;
  uint32_t want_large;      // record large gaps
  uint32_t large_min_gap;   // 0: the reference's rule (gap >= 500 or merit >= 10); else every gap >= it
  uint32_t b_mode;          // medium primes: 0 = thread per prime, 1 = lane per (prime, residue)
  const uint32_t* gbm;      // large-prime bitmap of the launch (nullptr: none); ANDed in at fill
  uint32_t scatter_first;   // primes with index >= this were applied by the pre-pass
  uint32_t* tile_counter;
  TilePartial* partials;
  unsigned long long* acc;  // n_intervals * kAccStride
  LargeGapDev* large;
  uint32_t* large_iv;       // interval of each large gap
  uint32_t* large_count;
  uint32_t large_cap;
  OverflowGap* over;
  uint32_t* over_count;
  uint32_t over_cap;
  uint32_t* error;
  // emit mode (voss_primes_range): primes written at out[tile_offset[t] + rank]
  const unsigned long long* tile_offset;
  unsigned long long* out;
  unsigned long long out_cap;
};

// Host-callable launchers (sieve_kernels.cu).
struct LaunchShape {
  int grid;
  int block;
  size_t smem;
};
size_t sieve_smem_bytes(uint32_t tile_words);
int launch_sieve_stats(const SieveArgs& a, int grid, int block, size_t smem, void* stream);
int launch_sieve_emit(const SieveArgs& a, int grid, int block, size_t smem, void* stream);
int launch_stitch(const SieveArgs& a, void* stream);
int launch_reduce(const SieveArgs& a, IntervalOut* out, void* stream);
}  // namespace voss
struct voss_interval_stats;
namespace voss {
// out_index (nullptr: identity) gives each launch interval's position in `out`.
int launch_interval_finalize(const SieveArgs& a, const IntervalOut* io, voss_interval_stats* out,
                             const uint32_t* out_index, void* stream);
// Short intervals by Miller-Rabin (short_iv.cu): candidates into d_cand (n_cand), verdicts into
// d_ok, the work list and its counters in d_work / d_nwork, results at d_out[out_index].
int launch_short_intervals(const ShortInterval* d_iv, uint32_t n_iv, uint64_t n_cand, uint64_t* d_cand,
                           uint8_t* d_ok, uint32_t* d_work, uint32_t* d_nwork, voss_interval_stats* d_out,
                           int sm_count, void* stream);
int launch_scatter_large(const uint32_t* primes, const uint64_t* magic, uint32_t j0, uint32_t j1,
                         const IntervalScatter* iv, uint32_t n_iv, uint32_t* gbm, int sm_count, void* stream);
int sieve_kernel_attrs(int block, size_t smem, int* max_ctas_per_sm);
// Large-gap list sorted by position on the device (large_sort.cu): keys and idx hold 2n entries.
size_t large_sort_temp_bytes(uint32_t n, int end_bit);
int launch_large_sort(const LargeGapDev* in, uint32_t n, int end_bit, unsigned long long* keys, uint32_t* idx,
                      void* temp, size_t temp_bytes, LargeGapDev* out, int sm_count, void* stream);
void build_presieve_tables(uint32_t* out /* kPreWords */);
int probe_smem_rmw(int sm_count, void* stream, float* ms, double* bytes);

// Miller-Rabin (mr_kernels.cu).  d_work holds count entries, d_nwork two counters (cleared here).
int launch_mr(const uint64_t* d_n, uint64_t count, uint8_t* d_out, uint32_t* d_work,
              uint32_t* d_nwork, void* stream, int sm_count);
// Gap proofs: endpoints (into d_ends / d_ends_ok, 2 * count each) through the Miller-Rabin
// kernels (work list d_work, counter d_nwork), then the interiors; count < 2^31.
int launch_prove_gaps(const uint64_t* d_p_after, const int32_t* d_gap, uint64_t count, uint8_t* d_ok,
                      uint64_t* d_ends, uint8_t* d_ends_ok, uint32_t* d_work, uint32_t* d_nwork, void* stream,
                      int sm_count);
// Montgomery products per second of independent squaring chains (moduli above / below 2^63).
int probe_mulmod(int sm_count, void* stream, double* full_per_s, double* small_per_s);

}  // namespace voss

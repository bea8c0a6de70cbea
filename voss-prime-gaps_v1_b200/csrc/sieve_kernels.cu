// sieve_kernels.cu — the sm_100a sieve-and-gap kernels.
//
// One persistent kernel (sieve_tiles_kernel) replaces the reference's per-segment pipeline
// memset -> graph of one sieve_w30_seg_kernel launch per base prime -> extract -> thrust::sort
// -> mod4 -> modq -> gaps (src/voss_v7_live.cu:120-312, 480-585).  Each CTA claims tiles of the
// wheel-30 bitmap from an atomic work counter and, for every tile, entirely in shared memory:
//   1. fill:     writes the tile pre-sieved by 7..31 from four periodic word-mask tables and
//                masks the interval's ends (the reference's cudaMemset + first-word patch, :496-500);
//   2. sieve:    clears the odd multiples of the base primes 37 <= p <= isqrt(hi-1)
//                (the reference's sieve_w30_seg_kernel, :120-143, one launch per prime):
//                  small primes  p <  tile_bytes/coop_div : one warp per prime: below
//                                                            tile_bytes/512 each residue progression
//                                                            split over all lanes in blocks of 4
//                                                            hits (no bank conflicts), above it 4
//                                                            lanes per residue,
//                  medium primes p <  mult_factor*tile_bytes: one thread per prime, 8 residues,
//                  large primes  otherwise                 : one thread per prime, walking its
//                                                            multiples across the tile's span;
//   3. restore:  sets the bits of base primes lying in the tile (the reference starts each prime
//                at p^2, :452-466; here the p*1 hit is undone instead);
//   4. extract:  the residue classes for mod-4 and mod-q (:181-232) are counted by word (all
//                words w = c mod 1001 share their class slots); then each thread walks an equal
//                share of the tile's primes in order (ffs), its predecessor prime coming from a
//                block-wide max-scan of the chunks' last primes, and updates shared-memory
//                counters: the gap histogram (:278-280), the per-residue gap histogram (:282-287),
//                the large-gap list (:289-299) and the tile's maximal gap.  Primes never reach HBM.
// The gaps across tile seams are added by stitch_kernel; reduce_kernel gives each interval its
// first/last prime and maximal gap.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "voss.h"
#include "voss_internal.h"

namespace voss {

// [bi*8 + o]: for a prime p = 30a + b (b = W30[bi]) and multiplier residue w = W30[o],
// p*w = 30*(a*w + D) + W30[B] with D = floor(b*w/30), stored as D | (B << 5).
__constant__ uint8_t c_wheel_step[64];
// residue r (mod 30) -> wheel bit index, or -1 when gcd(r, 30) > 1.
__constant__ int8_t c_res_bit[32];
// Wheel walk of a prime p = 30a + W30[bi] over its multiples p*m with gcd(m, 30) = 1.
// [bi*30 + t]: t = (offset of the first multiple of p at or above a tile's start) mod 30 gives
// m mod 30 = t * p^-1 (mod 30); stored: (steps to the next m coprime to 30) | (its wheel index << 3).
__constant__ uint8_t c_walk_start[240];
// [bi*8 + j]: from m = 30c + W30[j] to the next coprime m, the byte index of p*m grows by
// a*gap_j + corr (gap_j = W30[j+1] - W30[j], W30[8] = 31); stored: .x = ~(1 << bit of p*m)
// (rotated left by 8 * (byte & 3) it is the clear mask of that byte's lane in its word; the
// funnel shift takes its count mod 32, so byte << 3 is that rotation),
// .y = gap_j | corr << 16.
__constant__ uint2 c_walk_step[64];
// The same steps packed into registers for the tile kernel's walk (no table load per visit:
// shared-memory wavefronts are as scarce as issue slots there): nibble j of [bi] is corr_j,
// nibble j of [8 + bi] the bit of p*m, nibble j of kGap2Packed gap_j / 2; the walk rotates the
// three words by 4 bits per step, so the current step is always nibble 0.
__constant__ uint32_t c_walk_pk[16];
constexpr uint32_t kGap2Packed = 0x13212123u;

static int ensure_tables();

// Constant memory is per device: the tables are uploaded once for each device ordinal.
static std::atomic<uint64_t> g_tables_ready{0};

__device__ __forceinline__ uint32_t w30(uint32_t o) {
  return (uint32_t)((kW30Packed >> (8u * o)) & 0xFFu);
}

// x mod p with m = floor((2^64-1)/p): q <= x/p < q + 3.
__device__ __forceinline__ uint32_t mod_barrett(uint64_t x, uint32_t p, uint64_t m) {
  uint64_t q = __umul64hi(x, m);
  uint64_t r = x - q * (uint64_t)p;
  if (r >= p) r -= p;
  if (r >= p) r -= p;
  return (uint32_t)r;
}

// x mod p for x < 2^53 and 8 <= p < 2^30 from the Barrett constant m = floor((2^64-1)/p), with
// xs = x * 2^-64 as a double (exact).  m rounded to double times xs is x/p within a relative
// 2^-53 (x/p < 2^50), so adding 2^52 in the same rounding (fma) leaves an integer q within 0.63
// of x/p in the low mantissa bits; x - q p then lies in (-p, 2p), which its low 32 bits hold.
__device__ __forceinline__ uint32_t mod_by_magic_fma(uint64_t x, double xs, uint32_t p, uint64_t m) {
  const double qd = __fma_rn(xs, __ull2double_rn(m), 4503599627370496.0);
  uint32_t r = (uint32_t)x - (uint32_t)__double2loint(qd) * p;
  r += (int32_t)r < 0 ? p : 0u;
  r -= r >= p ? p : 0u;
  return r;
}

// x mod p from a double-precision estimate of the quotient, for p >= 2^11 and x < 2^62:
// xd = x and inv = 1/p rounded to double, so xd * inv is within (x/p) * 3 * 2^-53 < 2^-1 of x/p
// and its truncation is floor(x/p) - 1, floor(x/p) or floor(x/p) + 1; one signed correction
// finishes the remainder.
__device__ __forceinline__ uint32_t mod_by_estimate(uint64_t x, double xd, uint32_t p, double inv) {
  const uint64_t q = __double2ull_rz(xd * inv);
  int64_t r = (int64_t)(x - q * (uint64_t)p);
  if (r < 0) r += p;
  else if (r >= (int64_t)p) r -= p;
  return (uint32_t)r;
}

__device__ __forceinline__ uint64_t isqrt_u64(uint64_t x) {
  uint64_t s = (uint64_t)sqrt((double)x);
  if (s > 0xFFFFFFFFull) s = 0xFFFFFFFFull;
  while (s * s > x) --s;
  while (s < 0xFFFFFFFFull && (s + 1) * (s + 1) <= x) ++s;
  return s;
}

// number of table primes <= v
__device__ __forceinline__ uint32_t count_le(const uint32_t* pr, uint32_t n, uint64_t v) {
  if (v >= 0xFFFFFFFFull) return n;
  uint32_t lo = 0, hi = n, x = (uint32_t)v;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (pr[mid] <= x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// number of table primes < v
__device__ __forceinline__ uint32_t count_lt(const uint32_t* pr, uint32_t n, uint64_t v) {
  if (v == 0) return 0;
  return count_le(pr, n, v - 1);
}

// number of table primes <= v, found by the 32 lanes of a warp together: each round probes 32
// evenly spaced entries of the remaining range and keeps the slice between the last probe <= v
// and the first > v, so a table of n primes takes about log32(n) rounds of loads instead of
// log2(n) dependent ones.  Every lane returns the count.
__device__ __forceinline__ uint32_t count_le_warp(const uint32_t* pr, uint32_t n, uint64_t v, uint32_t lane) {
  if (v >= 0xFFFFFFFFull) return n;
  const uint32_t x = (uint32_t)v;
  uint32_t lo = 0, hi = n;  // the count lies in [lo, hi]
  while (hi - lo > 32u) {
    const uint32_t step = (hi - lo + 31u) >> 5;
    const uint32_t pos = lo + lane * step;
    const bool le = pos < hi && pr[pos] <= x;
    const uint32_t k = (uint32_t)__popc(__ballot_sync(0xFFFFFFFFu, le));  // probes 0..k-1 are <= x
    const uint32_t nlo = k ? lo + (k - 1u) * step + 1u : lo;
    const uint32_t bound = lo + k * step;  // the first probe > x, when it exists
    if (bound < hi) hi = bound;
    lo = nlo;
  }
  const bool le = lo + lane < hi && pr[lo + lane] <= x;
  return lo + (uint32_t)__popc(__ballot_sync(0xFFFFFFFFu, le));
}

__device__ __forceinline__ uint32_t count_lt_warp(const uint32_t* pr, uint32_t n, uint64_t v, uint32_t lane) {
  return v == 0 ? 0u : count_le_warp(pr, n, v - 1, lane);
}

__device__ __forceinline__ uint32_t find_interval(const SieveArgs& a, uint32_t t) {
  if (a.tile_iv) return a.tile_iv[t];  // the launch's tile -> interval table
  uint32_t lo = 0, hi = a.n_intervals;  // largest i with tile_begin <= t
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (a.iv[mid].tile_begin <= t) lo = mid; else hi = mid;
  }
  return lo;
}

#ifdef VOSS_BOUNDS_CHECK
#define VOSS_SM_GUARD(idx, limit)             \
  if ((idx) >= (limit)) {                     \
    atomicOr(err, kErrBounds);                \
    return;                                   \
  }
#else
#define VOSS_SM_GUARD(idx, limit)
#endif

__device__ __forceinline__ void clear_bit_word(uint32_t* bm, uint32_t word, uint32_t mask,
                                               uint32_t limit, uint32_t* err) {
  VOSS_SM_GUARD(word, limit)
  atomicAnd(bm + word, mask);
}

// Clears bit `bit` of every byte start, start + 4 ws, start + 8 ws, ... below Lt (one lane of a
// warp-cooperative small prime; the stride is 4 ws bytes = ws words).  The stride is a multiple of
// 4 bytes, so the byte lane inside the word, and with it the mask, never changes; four clears per
// loop trip.
__device__ __forceinline__ void clear_lane_progression(uint32_t* bm, uint32_t start, uint32_t ws,
                                                       uint32_t bit, uint32_t Lt, uint32_t nw,
                                                       uint32_t* err) {
  const uint32_t mask = ~(1u << (((start & 3u) << 3) | bit));
  const uint32_t wlim = (Lt + 3u - (start & 3u)) >> 2;  // start + 4k < Lt  <=>  (start >> 2) + k < wlim
  uint32_t w = start >> 2;
  if (wlim > 3u * ws) {
    const uint32_t wlim4 = wlim - 3u * ws;
#pragma unroll 2
    for (; w < wlim4; w += 4u * ws) {
      clear_bit_word(bm, w, mask, nw, err);
      clear_bit_word(bm, w + ws, mask, nw, err);
      clear_bit_word(bm, w + 2u * ws, mask, nw, err);
      clear_bit_word(bm, w + 3u * ws, mask, nw, err);
    }
  }
  for (; w < wlim; w += ws) clear_bit_word(bm, w, mask, nw, err);
}

// One lane's share of a warp-cooperative residue progression bytes s, s + p, s + 2p, ... (p odd):
// lane m clears the hits 4m + 128t + u (u = 0..3, t >= 0), i.e. bytes
// byte + u p + 128 p t with byte = s + 4 p m, all below Lt.  For a fixed (t, u) the 32 lanes'
// words are c + p m + 32 p t with c = (s + u p) >> 2 common to the warp: as p is odd they fall
// in 32 distinct banks, so every shared-memory atomic of the warp is a single wavefront.  The
// lane's four bytes of a block lie in four distinct byte lanes of their words and a block
// advances by 128 p bytes = 32 p words, so the four masks and word offsets stay fixed.
__device__ __forceinline__ void clear_block_progression(uint32_t* bm, uint32_t byte, uint32_t p, uint32_t bit,
                                                        uint32_t Lt, uint32_t nw, uint32_t* err) {
  if (byte + 3u * p < Lt) {
    const uint32_t b1 = byte + p, b2 = b1 + p, b3 = b2 + p;
    // ~(1 << bit) rotated to each byte's lane (the funnel shift takes its count mod 32)
    const uint32_t nb = ~(1u << bit);
    const uint32_t m0 = __funnelshift_l(nb, nb, byte << 3), m1 = __funnelshift_l(nb, nb, b1 << 3);
    const uint32_t m2 = __funnelshift_l(nb, nb, b2 << 3), m3 = __funnelshift_l(nb, nb, b3 << 3);
    uint32_t w0 = byte >> 2;
    const uint32_t d1 = (b1 >> 2) - w0, d2 = (b2 >> 2) - w0, d3 = (b3 >> 2) - w0;
    const uint32_t ws = 32u * p;
    // b3 + 128 p k < Lt  <=>  (b3 >> 2) + 32 p k < lim
    const uint32_t lim = ((Lt + 3u - (b3 & 3u)) >> 2) - d3;
    uint32_t k = 0;
#pragma unroll 4
    for (; w0 < lim; w0 += ws, ++k) {
      clear_bit_word(bm, w0, m0, nw, err);
      clear_bit_word(bm, w0 + d1, m1, nw, err);
      clear_bit_word(bm, w0 + d2, m2, nw, err);
      clear_bit_word(bm, w0 + d3, m3, nw, err);
    }
    byte += 128u * p * k;
  }
  // at most three hits remain (byte + 3p >= Lt); the next block belongs to the next lane
  {
    const uint32_t nb = ~(1u << bit);  // rotated by 8 * (byte & 3): the funnel shift takes byte << 3 mod 32
    for (; byte < Lt; byte += p) clear_bit_word(bm, byte >> 2, __funnelshift_l(nb, nb, byte << 3), nw, err);
  }
}

// Clears bit `bit` of bytes byte, byte + p, byte + 2p, ... below Lt (p odd).  Four consecutive
// hits fall in the four distinct byte lanes of their words, and advancing all four by 4p bytes
// moves each by exactly p words, so the unrolled loop keeps four fixed masks and word offsets.
__device__ __forceinline__ void clear_progression(uint32_t* bm, uint32_t byte, uint32_t p, uint32_t bit,
                                                  uint32_t Lt, uint32_t nw, uint32_t* err) {
  if (byte + 3u * p < Lt) {
    // the four hits' byte lanes are j0, j0 + p, j0 + 2p, j0 + 3p (mod 4): one lane up each time
    // for p = 1 (mod 4), one lane down for p = 3, so each mask is the previous one rotated by a byte
    const uint32_t j0 = byte & 3u;
    const uint32_t nb = ~(1u << bit);
    const uint32_t rot = (p & 2u) ? 24u : 8u;
    const uint32_t m0 = __funnelshift_l(nb, nb, byte << 3), m1 = __funnelshift_l(m0, m0, rot),
                   m2 = __funnelshift_l(m1, m1, rot), m3 = __funnelshift_l(m2, m2, rot);
    uint32_t w0 = byte >> 2;
    const uint32_t d1 = (j0 + p) >> 2, d2 = (j0 + 2u * p) >> 2, d3 = (j0 + 3u * p) >> 2;
    // b3 + 4pk < Lt  <=>  w0 + k < lim  (w0 + d3 = b3 >> 2)
    const uint32_t lim = ((Lt + 3u - ((j0 + 3u * p) & 3u)) >> 2) - d3;
    for (; w0 < lim; w0 += p) {
      clear_bit_word(bm, w0, m0, nw, err);
      clear_bit_word(bm, w0 + d1, m1, nw, err);
      clear_bit_word(bm, w0 + d2, m2, nw, err);
      clear_bit_word(bm, w0 + d3, m3, nw, err);
    }
    byte = (w0 << 2) | j0;  // the loop advanced by 4p bytes (p words) per trip
  }
  {
    const uint32_t nb = ~(1u << bit);  // rotated by 8 * (byte & 3): the funnel shift takes byte << 3 mod 32
    for (; byte < Lt; byte += p) clear_bit_word(bm, byte >> 2, __funnelshift_l(nb, nb, byte << 3), nw, err);
  }
}

// Clears every multiple p*m (gcd(m, 30) = 1) of prime p = 30a + W30[bi] in the tile whose first
// integer is vbase (a multiple of 30) and whose length is Lt bytes, visiting only those multiples
// (about 8*Lt/p of them) instead of eight residue progressions.  rv = vbase mod p.
__device__ __forceinline__ void clear_wheel_walk(uint32_t* bm, uint32_t p, uint32_t a, uint32_t bi, uint32_t rv,
                                                 const uint8_t* s_wstart, const uint2* s_wpk,
                                                 uint32_t Lt, uint32_t nw, uint32_t* err) {
  uint32_t off = rv ? p - rv : 0u;         // first multiple of p at or above vbase, as an offset
  const uint32_t t = off - 30u * (off / 30u);
  const uint32_t st = s_wstart[bi * 30u + t];
  off += (st & 7u) * p;                     // first multiple with m coprime to 30
  const uint32_t sh = 4u * (st >> 3);
  uint32_t byte = off / 30u;
  const uint2 cb = s_wpk[bi];
  const uint32_t c0 = cb.x, b0 = cb.y;
  uint32_t G = __funnelshift_r(kGap2Packed, kGap2Packed, sh);
  uint32_t C = __funnelshift_r(c0, c0, sh), B = __funnelshift_r(b0, b0, sh);
  const uint32_t a2 = 2u * a;
  while (byte < Lt) {
    // ~(1 << bit) rotated by 8 * (byte & 3): the funnel shift takes its count mod 32, and
    // bit < 8 leaves the byte-lane part of (byte << 3) + bit untouched
    clear_bit_word(bm, byte >> 2, __funnelshift_l(0xFFFFFFFEu, 0xFFFFFFFEu, ((byte << 3) & 24u) | (B & ~24u)), nw, err);
    byte += a2 * (G & 3u) + (C & 7u);
    G = __funnelshift_r(G, G, 4);
    C = __funnelshift_r(C, C, 4);
    B = __funnelshift_r(B, B, 4);
  }
}

__device__ __forceinline__ void sm_add(uint32_t* cnt, uint32_t idx, uint32_t* err) {
  VOSS_SM_GUARD(idx, (uint32_t)kSmCounters)
  atomicAdd(cnt + idx, 1u);
}

__device__ __forceinline__ void sm_add_n(uint32_t* cnt, uint32_t idx, uint32_t v, uint32_t* err) {
  VOSS_SM_GUARD(idx, (uint32_t)kSmCounters)
  atomicAdd(cnt + idx, v);
}

// Carry-save adder over bit planes: l = a ^ b ^ c, h = majority(a, b, c).
__device__ __forceinline__ void csa(uint32_t& h, uint32_t& l, uint32_t a, uint32_t b, uint32_t c) {
  const uint32_t u = a ^ b;
  h = (a & b) | (u & c);
  l = u ^ c;
}

// Swaps the bits of x selected by mask << s with the bits of y selected by mask (one step of an
// 8x8 bit-matrix transpose applied to the four byte lanes at once).
__device__ __forceinline__ void swap_bits(uint32_t& x, uint32_t& y, uint32_t mask, uint32_t s) {
  const uint32_t t = ((x >> s) ^ y) & mask;
  y ^= t;
  x ^= t << s;
}

// The residue-class counters of a tile's primes (k mod 28 and k mod 143 by wheel residue: every
// q of the reference's mod-4 and mod-q counts, voss_v7_live.cu:181-232), counted by word instead
// of by prime.  The slots of bit b of word w are 8 ((k28 + 4w) mod 28) + b and
// 8 ((k143 + 4w) mod 143) + b, and 4004 = 4 * 1001 is a multiple of 28 and of 143, so all words
// w = c (mod 1001) share their 32 slots in each block.  A thread takes the words of one class c
// and adds them column by column into six bit planes with carry-save adders (a column counts at
// most 63 words; shared memory holds tiles of at most about 52,000 words, at most 52 per class),
// transposes the planes into 32 byte-sized column counts and adds each column to its two slots:
// 64 shared-memory atomics per class instead of two per prime.  The planes are first rotated by
// the lane number, so lane l adds column (s + l) mod 32 at step s: the k mod 28 slots of a warp
// then lie in 32 distinct banks (8 (k28 + 4w) mod 32 is the same for every w), and the k mod 143
// slots as well once each lane's bytes are shifted by its own (k143 + 4c) mod 4.
template <int BLOCK>
__device__ __forceinline__ void class_counts_by_word(const uint32_t* bm, uint32_t nw, uint32_t k28,
                                                     uint32_t k143, uint32_t* cnt, uint32_t lane,
                                                     uint32_t* err) {
  for (uint32_t c = threadIdx.x; c < 1001u; c += BLOCK) {
    uint32_t p0 = 0, p1 = 0, p2 = 0, p3 = 0, p4 = 0, p5 = 0;
    uint32_t w = c;
    for (; w + 7u * 1001u < nw; w += 8u * 1001u) {  // eight words: three levels of adders
      uint32_t a1, a2, a3, a4, b1, b2, c1;
      csa(a1, p0, p0, bm[w], bm[w + 1001u]);
      csa(a2, p0, p0, bm[w + 2u * 1001u], bm[w + 3u * 1001u]);
      csa(b1, p1, p1, a1, a2);
      csa(a3, p0, p0, bm[w + 4u * 1001u], bm[w + 5u * 1001u]);
      csa(a4, p0, p0, bm[w + 6u * 1001u], bm[w + 7u * 1001u]);
      csa(b2, p1, p1, a3, a4);
      csa(c1, p2, p2, b1, b2);
      const uint32_t t3 = p3 & c1;
      p3 ^= c1;
      p5 ^= p4 & t3;
      p4 ^= t3;
    }
    for (; w < nw; w += 1001u) {  // the rest one word at a time
      const uint32_t x = bm[w];
      const uint32_t t0 = p0 & x;
      p0 ^= x;
      const uint32_t t1 = p1 & t0;
      p1 ^= t0;
      const uint32_t t2 = p2 & t1;
      p2 ^= t1;
      const uint32_t t3 = p3 & t2;
      p3 ^= t2;
      p5 ^= p4 & t3;
      p4 ^= t3;
    }
    // rotate: bit s of each plane becomes column (s + lane) mod 32
    p0 = __funnelshift_r(p0, p0, lane);
    p1 = __funnelshift_r(p1, p1, lane);
    p2 = __funnelshift_r(p2, p2, lane);
    p3 = __funnelshift_r(p3, p3, lane);
    p4 = __funnelshift_r(p4, p4, lane);
    p5 = __funnelshift_r(p5, p5, lane);
    // transpose each byte lane's 8x8 bit matrix (planes 6 and 7 are zero): afterwards byte n of
    // t_j is the count of rotated column 8n + j
    uint32_t t0 = p0, t1 = p1, t2 = p2, t3 = p3, t4 = p4, t5 = p5, t6 = 0, t7 = 0;
    swap_bits(t0, t4, 0x0F0F0F0Fu, 4);
    swap_bits(t1, t5, 0x0F0F0F0Fu, 4);
    swap_bits(t2, t6, 0x0F0F0F0Fu, 4);
    swap_bits(t3, t7, 0x0F0F0F0Fu, 4);
    swap_bits(t0, t2, 0x33333333u, 2);
    swap_bits(t1, t3, 0x33333333u, 2);
    swap_bits(t4, t6, 0x33333333u, 2);
    swap_bits(t5, t7, 0x33333333u, 2);
    swap_bits(t0, t1, 0x55555555u, 1);
    swap_bits(t2, t3, 0x55555555u, 1);
    swap_bits(t4, t5, 0x55555555u, 1);
    swap_bits(t6, t7, 0x55555555u, 1);
    const uint32_t tt[8] = {t0, t1, t2, t3, t4, t5, t6, t7};
    const uint32_t u28 = (k28 + 4u * c) % 28u, u143 = (k143 + 4u * c) % 143u;
    const uint32_t base28 = (uint32_t)kSmCls28 + 8u * u28, base143 = (uint32_t)kSmCls143 + 8u * u143;
    // k mod 143 slots: byte n of the step's word is taken from byte (n - m) mod 4, m = u143 mod 4,
    // so that lane l adds column (s + l - 8m) mod 32 there
    const uint32_t m = u143 & 3u;
    const uint32_t r143 = (lane - 8u * m) & 31u;
    uint32_t sel[4];
#pragma unroll
    for (uint32_t n = 0; n < 4; ++n) sel[n] = 0x4440u | ((n - m) & 3u);
#pragma unroll
    for (uint32_t s = 0; s < 32; ++s) {
      const uint32_t v28 = (tt[s & 7u] >> (8u * (s >> 3))) & 0xFFu;
      const uint32_t v143 = __byte_perm(tt[s & 7u], 0u, sel[s >> 3]);
      sm_add_n(cnt, base28 + ((s + lane) & 31u), v28, err);
      sm_add_n(cnt, base143 + ((s + r143) & 31u), v143, err);
    }
  }
}

// Mask of the bits of word w whose integers lie in [vlo, vhi); v0 = value of byte 4w, residue 0.
__device__ __forceinline__ uint32_t edge_mask(uint64_t v0, uint64_t vlo, uint64_t vhi) {
  uint32_t m = 0;
#pragma unroll
  for (uint32_t j = 0; j < 4; ++j)
#pragma unroll
    for (uint32_t o = 0; o < 8; ++o) {
      uint64_t v = v0 + 30u * j + w30(o);
      if (v >= vlo && v < vhi) m |= 1u << (8u * j + o);
    }
  return m;
}

__device__ __forceinline__ uint32_t pre_mod(int g) {
  return g == 0 ? 1001u : (g == 1 ? 323u : (g == 2 ? 667u : 31u));
}
__device__ __forceinline__ uint32_t pre_off(int g) {
  return g == 0 ? 0u : (g == 1 ? 1001u : (g == 2 ? 1324u : 1991u));
}

#ifdef VOSS_PHASE_TIMING
// Instrumented build only: per-phase cycles summed over all CTAs (thread 0 of each CTA
// timestamps every phase boundary after a block barrier).
__device__ unsigned long long g_phase_cycles[16];
#define VOSS_PHASE(k)                                  \
  __syncthreads();                                     \
  if (threadIdx.x == 0) {                              \
    const long long now__ = clock64();                 \
    ph_acc[(k)] += (unsigned long long)(now__ - ph_t); \
    ph_t = now__;                                      \
  }
#else
#define VOSS_PHASE(k)
#endif

struct TileHdr {  // one tile's header (double-buffered: the next tile's is built during this one)
  unsigned long long ktile, vbase, vlo, vhi, seg_k;
  uint32_t nw, lt, np, ia, ib, iw, vb, cthr, k28, k143;
  uint32_t pre_base[kPreGroups];
  uint32_t interval, tile;
  uint32_t r0, r1;       // base primes lying in the tile (restore)
  uint32_t coop_ctr, b_ctr, c_ctr;  // work counters of the three prime categories
  unsigned long long gword;         // the tile's first word in the large-prime bitmap
  uint32_t first;
};

struct CtaState {  // what a CTA carries from tile to tile
  uint32_t cur_iv, since_flush, flush;
  uint32_t c_lt, c_ia, c_ib, c_iw;  // category bounds over the whole table for tile length c_lt
  unsigned long long count_total;
};

template <int BLOCK>
struct BlockScratch {
  int32_t warp_max[BLOCK / 32];
  int32_t warp_prefix[BLOCK / 32];
  int32_t block_max;
  uint32_t warp_sum[BLOCK / 32];
  unsigned long long warp_key[BLOCK / 32];
};

// Exclusive max-scan of `v` over thread order; returns the exclusive prefix and, through
// *total, the max over the block.
template <int BLOCK>
__device__ __forceinline__ int32_t block_excl_max(int32_t v, BlockScratch<BLOCK>& S, int32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int32_t incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d) incl = max(incl, t);
  }
  if (lane == 31) S.warp_max[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int32_t x = lane < BLOCK / 32 ? S.warp_max[lane] : -1;
    int32_t y = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int32_t t = __shfl_up_sync(0xFFFFFFFFu, y, d);
      if (lane >= d) y = max(y, t);
    }
    int32_t ex = __shfl_up_sync(0xFFFFFFFFu, y, 1);
    if (lane == 0) ex = -1;
    if (lane < BLOCK / 32) S.warp_prefix[lane] = ex;
    if (lane == BLOCK / 32 - 1) S.block_max = y;
  }
  __syncthreads();
  int32_t ex = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
  if (lane == 0) ex = -1;
  ex = max(ex, S.warp_prefix[warp]);
  *total = S.block_max;
  return ex;
}

template <int BLOCK>
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t v, BlockScratch<BLOCK>& S, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) S.warp_sum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t x = lane < BLOCK / 32 ? S.warp_sum[lane] : 0;
    uint32_t y = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t t = __shfl_up_sync(0xFFFFFFFFu, y, d);
      if (lane >= d) y += t;
    }
    if (lane < BLOCK / 32) S.warp_sum[lane] = y - x;  // exclusive prefix of warps
    if (lane == BLOCK / 32 - 1) S.warp_prefix[0] = (int32_t)y;
  }
  __syncthreads();
  uint32_t ex = incl - v + S.warp_sum[warp];
  *total = (uint32_t)S.warp_prefix[0];
  return ex;
}

template <int BLOCK>
__device__ __forceinline__ void block_reduce_tile(uint32_t cnt, unsigned long long key,
                                                  BlockScratch<BLOCK>& S, uint32_t* cnt_total,
                                                  unsigned long long* key_max) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, d);
    unsigned long long k2 = __shfl_down_sync(0xFFFFFFFFu, key, d);
    key = k2 > key ? k2 : key;
  }
  if (lane == 0) {
    S.warp_sum[warp] = cnt;
    S.warp_key[warp] = key;
  }
  __syncthreads();
  if (warp == 0) {
    uint32_t c = lane < BLOCK / 32 ? S.warp_sum[lane] : 0;
    unsigned long long k = lane < BLOCK / 32 ? S.warp_key[lane] : 0ull;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      c += __shfl_down_sync(0xFFFFFFFFu, c, d);
      unsigned long long k2 = __shfl_down_sync(0xFFFFFFFFu, k, d);
      k = k2 > k ? k2 : k;
    }
    if (lane == 0) {
      *cnt_total = c;
      *key_max = k;
    }
  }
}

// Accumulator word of shared counter i.  The class counters fold: shared class c of the
// (k mod 28) block is class c mod 28, of the (k mod 143) block class c mod 143.
__device__ __forceinline__ uint32_t acc_index(uint32_t i) {
  if (i < (uint32_t)kSmModq) return (uint32_t)kAccHist + i;
  if (i < (uint32_t)kSmCls28) {
    const uint32_t j = i - (uint32_t)kSmModq;  // 8 * bin + residue
    return (uint32_t)kAccModq + (j & 7u) * (uint32_t)kModqBins + (j >> 3);
  }
  if (i < (uint32_t)kSmCls143) {
    const uint32_t c = (i - (uint32_t)kSmCls28) >> 3;
    return (uint32_t)kAccCls28 + 8u * (c >= 28u ? c - 28u : c) + (i & 7u);
  }
  const uint32_t c = (i - (uint32_t)kSmCls143) >> 3;
  return (uint32_t)kAccCls143 + 8u * (c >= 143u ? c - 143u : c) + (i & 7u);
}

// Warp-cooperative primes p >= tile bytes / kSmallSplitDiv give each residue 4 lanes (their few
// hits per residue keep a lane's loop long); smaller ones give each residue all 32 lanes in turn.
#ifndef VOSS_SMALL_SPLIT_DIV
#define VOSS_SMALL_SPLIT_DIV 512
#endif
constexpr uint32_t kSmallSplitDiv = VOSS_SMALL_SPLIT_DIV;

constexpr uint32_t kFlushEvery = 2048;  // tiles between counter flushes (u32 headroom)

// The header of tile t, built by one warp: the lanes compute the same scalars and share the
// table searches (count_le_warp); lane 0 writes the header.  t >= n_tiles marks the end.
__device__ __forceinline__ void tile_header(TileHdr& H, CtaState& St, const SieveArgs& a, uint32_t t,
                                            uint32_t ln) {
  {
    {
      const uint32_t ivx = t < a.n_tiles ? find_interval(a, t) : kNone;
      if (ln == 0) {
        H.tile = t;
        H.interval = ivx;
      }
      if (t >= a.n_tiles) return;
      const IntervalDev iv = a.iv[ivx];
      const uint32_t tl = t - iv.tile_begin;
      const uint64_t wofs = (uint64_t)tl * a.tile_words;
      const uint64_t nw64 = iv.n_words - wofs;
      const uint32_t nw = nw64 < a.tile_words ? (uint32_t)nw64 : a.tile_words;
      const uint64_t ktile = iv.k0 + 4ull * wofs;
      const uint64_t vbase = 30ull * ktile;
      const uint32_t lt = 4u * nw;
      uint64_t vend = vbase + 30ull * lt;
      if (vend > iv.hi) vend = iv.hi;
      // table searches, skipped where the answer is known: a tile past the table's last prime
      // needs every prime and holds none of them; the category bounds over the whole table
      // depend only on the tile length (count_lt over np primes = min(that, np))
      const uint64_t sq = isqrt_u64(vend - 1);
      uint32_t np = sq >= a.p_max ? a.n_primes : count_le_warp(a.primes, a.n_primes, sq, ln);
      if (a.gbm && np > a.scatter_first) np = a.scatter_first;  // the rest came from the pre-pass
      if (lt != St.c_lt) {
        const uint32_t ia = count_lt_warp(a.primes, a.n_primes, (uint64_t)(lt / a.coop_div), ln);
        const uint32_t ib = count_lt_warp(a.primes, a.n_primes, (uint64_t)lt * a.mult_factor, ln);
        const uint32_t iw = count_lt_warp(a.primes, a.n_primes, ((uint64_t)lt * a.walk_sixteenths) >> 4, ln);
        __syncwarp();
        if (ln == 0) {
          St.c_ia = ia;
          St.c_ib = ib;
          St.c_iw = iw;
          St.c_lt = lt;
        }
        __syncwarp();
      }
      const uint32_t ia = min(St.c_ia, np);
      const uint32_t ib0 = min(St.c_ib, np);
      const uint32_t ib = ib0 < ia ? ia : ib0;
      const uint32_t iw0 = min(St.c_iw, np);
      const uint32_t iw = iw0 < ia ? ia : (iw0 > ib ? ib : iw0);
      uint32_t r0 = a.n_primes, r1 = a.n_primes;
      if (vbase <= a.p_max) {
        r0 = count_lt_warp(a.primes, a.n_primes, vbase, ln);
        r1 = count_lt_warp(a.primes, a.n_primes, vbase + 30ull * lt, ln);
      }
      if (ln == 0) {
        H.ktile = ktile;
        H.vbase = vbase;
        H.vlo = iv.lo;
        H.vhi = iv.hi;
        H.seg_k = iv.seg_k;
        H.nw = nw;
        H.lt = lt;
        H.np = np;
        H.gword = iv.gword + wofs;
        H.ia = ia;
        H.ib = ib;
        H.iw = iw;
        H.r0 = r0;
        H.r1 = r1;
        uint32_t vb = kNone;
        if (iv.seg_k) {
          uint64_t kb = (ktile / iv.seg_k + 1) * iv.seg_k;
          if (kb < ktile + lt) vb = (uint32_t)(30ull * (kb - ktile));
        }
        H.vb = vb;
        // large-gap candidates: g >= cthr, one tile-uniform threshold.  Reference rule
        // (voss_v7_live.cu:289-294): g > 100 and (g >= 500 or g / log(p) >= 10); no gap of the
        // tile below 10 log(vbase) - 3 can reach merit 10.  With large_min_gap: g >= large_min_gap.
        // (single-precision log: its error, a few units of 1e-6 relative at these sizes, is far
        // inside the margin of 3; the kept gaps are then decided by the double merit below)
        const float th = floorf(10.0f * __logf((float)(vbase > 7 ? vbase : 7))) - 3.0f;
        uint32_t gthr = th < 0.0f ? 0u : (uint32_t)th;
        gthr = gthr < 101u ? 101u : (gthr > 500u ? 500u : gthr);
        H.cthr = !a.want_large ? kNone : (a.large_min_gap ? a.large_min_gap : gthr);
        H.k28 = (uint32_t)(ktile % 28ull);
        H.k143 = (uint32_t)(ktile % 143ull);
        const uint64_t wt = ktile >> 2;
#pragma unroll
        for (int g = 0; g < kPreGroups; ++g) H.pre_base[g] = (uint32_t)(wt % pre_mod(g));
        H.coop_ctr = 0;
        H.b_ctr = 0;
        H.c_ctr = 0;
        H.first = kNone;
      }
    }
  }
}

template <int BLOCK, bool EMIT>
__global__ void __launch_bounds__(BLOCK, (BLOCK == 512 ? 2 : 1))
sieve_tiles_kernel(SieveArgs a) {
  extern __shared__ __align__(16) uint32_t smem[];
  uint32_t* bm = smem;
  uint32_t* pre = smem + a.tile_words;
  uint32_t* cnt = pre + kPreWords;
  __shared__ TileHdr HH[2];  // this tile's header and the next one's
  __shared__ CtaState St;
  __shared__ BlockScratch<BLOCK> S;
  // Wheel tables in shared memory: lanes index them by their own prime's residue, which
  // would serialize in the constant cache.
  __shared__ __align__(8) uint8_t s_step[64];
  __shared__ int8_t s_rb[32];
  __shared__ uint32_t s_pos[32];  // bit b of a word -> integer offset 30 * (b / 8) + W30[b % 8]
  __shared__ uint8_t s_wstart[240];
  __shared__ uint2 s_wpk[8];
  __shared__ uint32_t s_rank[EMIT ? 1 : BLOCK];   // first tile rank of each thread's chunk
  __shared__ int32_t s_before[EMIT ? 1 : BLOCK];  // last prime before each chunk (-1: none)
  __shared__ uint16_t s_mid[EMIT ? 1 : BLOCK];    // primes in the first C / 2 words of each chunk
  uint32_t* err = a.error;

  const int tid = threadIdx.x, lane = tid & 31;
  for (uint32_t i = tid; i < kPreWords; i += BLOCK) pre[i] = a.pretab[i];
  if (tid < 64) s_step[tid] = c_wheel_step[tid];
  if (tid < 32) s_rb[tid] = c_res_bit[tid];
  if (tid < 32) s_pos[tid] = 30u * ((uint32_t)tid >> 3) + w30((uint32_t)tid & 7u);
  if (tid < 240) s_wstart[tid] = c_walk_start[tid];
  if (tid < 8) s_wpk[tid] = make_uint2(c_walk_pk[tid], c_walk_pk[8 + tid]);
  if (!EMIT)
    for (uint32_t i = tid; i < (uint32_t)kSmCounters; i += BLOCK) cnt[i] = 0;
  if (tid == 0) {
    St.cur_iv = kNone;
    St.since_flush = 0;
    St.count_total = 0;
    St.c_lt = kNone;
  }
  __syncthreads();
  if (tid < 32) {  // the first tile: claim and header
    uint32_t t0 = 0;
    if (lane == 0) t0 = atomicAdd(a.tile_counter, 1u);
    tile_header(HH[0], St, a, __shfl_sync(0xFFFFFFFFu, t0, 0), (uint32_t)lane);
  }
  __syncthreads();
  uint32_t cur = 0;

  const uint32_t C = a.chunk_words;
#ifdef VOSS_PHASE_TIMING
  unsigned long long ph_acc[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  long long ph_t = clock64();
#endif

  for (;;) {
    TileHdr& H = HH[cur];  // built during the previous tile (or before the loop)
    // ---- flush ------------------------------------------------------------------------
    if (tid == 0) {
      const uint32_t ivx = H.tile < a.n_tiles ? H.interval : kNone;
      St.flush = (!EMIT && St.cur_iv != kNone &&
                  (ivx != St.cur_iv || St.since_flush >= kFlushEvery)) ? 1u : 0u;
    }
    __syncthreads();
    if (St.flush) {
      unsigned long long* acc = a.acc + (size_t)St.cur_iv * kAccStride;
      for (uint32_t i = tid; i < (uint32_t)kSmCounters; i += BLOCK) {
        uint32_t v = cnt[i];
        if (v) {
          atomicAdd(acc + acc_index(i), (unsigned long long)v);
          cnt[i] = 0;
        }
      }
      if (tid == 0) {
        atomicAdd(acc + kAccCount, St.count_total);
        St.count_total = 0;
        St.since_flush = 0;
      }
      __syncthreads();
    }
    if (H.tile >= a.n_tiles) break;
    if (tid == 0) St.cur_iv = H.interval;
    VOSS_PHASE(0)

    VOSS_PHASE(1)

    const uint32_t nw = H.nw, Lt = H.lt;

    // ---- 1. fill ----------------------------------------------------------------------
    {
      uint32_t ix[kPreGroups], st[kPreGroups];
#pragma unroll
      for (int g = 0; g < kPreGroups; ++g) {
        ix[g] = (H.pre_base[g] + (uint32_t)tid) % pre_mod(g);
        st[g] = (uint32_t)BLOCK % pre_mod(g);
      }
      const uint64_t vbase = H.vbase, vlo = H.vlo, vhi = H.vhi;
      const uint32_t* gbm = a.gbm ? a.gbm + H.gword : nullptr;
      // words [w_in, w_out) lie wholly inside [vlo, vhi) (v0 + 1 >= vlo and v0 + 120 <= vhi):
      // only the others need an edge mask
      const uint64_t lo_words = vlo <= vbase + 1 ? 0ull : (vlo - vbase + 118ull) / 120ull;
      const uint64_t hi_words = vhi < vbase + 120 ? 0ull : (vhi - vbase) / 120ull;
      const uint32_t w_in = (uint32_t)(lo_words < a.tile_words ? lo_words : a.tile_words);
      const uint32_t w_out = (uint32_t)(hi_words < a.tile_words ? hi_words : a.tile_words);
#pragma unroll 4
      for (uint32_t w = tid; w < a.tile_words; w += BLOCK) {
        uint32_t m = 0;
        if (w < nw) {
          m = pre[ix[0]] & pre[1001u + ix[1]] & pre[1324u + ix[2]] & pre[1991u + ix[3]];
          if (gbm) m &= gbm[w];
          if (w < w_in || w >= w_out) m &= edge_mask(vbase + 120ull * w, vlo, vhi);
        }
        bm[w] = m;
#pragma unroll
        for (int g = 0; g < kPreGroups; ++g) {
          ix[g] += st[g];
          if (ix[g] >= pre_mod(g)) ix[g] -= pre_mod(g);
        }
      }
    }
    __syncthreads();
    VOSS_PHASE(2)

    // Warp 0 claims the next tile and builds its header now, while the other warps start on
    // this tile's small primes (claimed dynamically, so they take over warp 0's share): the
    // header's dependent loads no longer hold the whole CTA at a barrier between tiles.
    if (tid < 32) {
      uint32_t tn = 0;
      if (lane == 0) tn = atomicAdd(a.tile_counter, 1u);
      tile_header(HH[cur ^ 1u], St, a, __shfl_sync(0xFFFFFFFFu, tn, 0), (uint32_t)lane);
    }

    // ---- 2. sieve ----------------------------------------------------------------------
    {
      const uint64_t ktile = H.ktile;
      const uint32_t ia = H.ia, ib = H.ib, iw = H.iw, np = H.np;
      // tiles below 2^53 reduce the prime offsets with one fma instead of the 64-bit Barrett product
      const bool fma_mod = H.vbase < (1ull << 53);
      const double ks = (double)ktile * 0x1p-64, vs = (double)H.vbase * 0x1p-64;
      // small primes: a warp per prime
      const uint32_t split = Lt / kSmallSplitDiv;
      const uint32_t lane_ofs = 4u * (uint32_t)lane;
      for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(&H.coop_ctr, 1u);
        i = __shfl_sync(0xFFFFFFFFu, i, 0);
        if (i >= ia) break;
        const uint32_t p = a.primes[i];
        const uint64_t m = a.magic[i];
        const uint32_t r = fma_mod ? mod_by_magic_fma(ktile, ks, p, m) : mod_barrett(ktile, p, m);
        const uint32_t pa = p / 30u, bi = (uint32_t)s_rb[p - 30u * pa];
        if (p >= split) {
          // 4 lanes per residue progression (lane = 4 o + q: bytes s_o + q p + 4p k)
          const uint32_t o = (uint32_t)lane >> 2;
          const uint32_t e = s_step[bi * 8u + o];
          const uint32_t delta = pa * w30(o) + (e & 31u);
          const uint32_t s = delta >= r ? delta - r : delta + p - r;
          clear_lane_progression(bm, s + ((uint32_t)lane & 3u) * p, p, e >> 5, Lt, nw, err);
        } else {
          // the eight residue progressions in turn, each split over all lanes in blocks of four
          // consecutive hits (bank-conflict-free, clear_block_progression)
          const uint32_t lp = lane_ofs * p;
#pragma unroll 1
          for (uint32_t o = 0; o < 8; ++o) {
            const uint32_t e = s_step[bi * 8u + o];
            const uint32_t delta = pa * w30(o) + (e & 31u);
            const uint32_t s = delta >= r ? delta - r : delta + p - r;
            clear_block_progression(bm, s + lp, p, e >> 5, Lt, nw, err);
          }
        }
      }
      VOSS_PHASE(3)
      // medium primes
      if (a.b_mode == 0) {
        // a thread per prime, 8 residue progressions; warps claim 32 consecutive primes at a time
        for (;;) {
          uint32_t base = 0;
          if (lane == 0) base = atomicAdd(&H.b_ctr, 32u);
          base = __shfl_sync(0xFFFFFFFFu, base, 0);
          if (base >= ib - ia) break;
          const uint32_t i = ia + base + (uint32_t)lane;
          if (i >= iw && i < ib) {
            // few hits per tile: walk the prime's coprime multiples
            const uint32_t p = a.primes[i];
            const uint32_t pa = p / 30u, bi = (uint32_t)s_rb[p - 30u * pa];
            const uint64_t m = a.magic[i];
            clear_wheel_walk(bm, p, pa, bi, fma_mod ? mod_by_magic_fma(H.vbase, vs, p, m) : mod_barrett(H.vbase, p, m),
                             s_wstart, s_wpk, Lt, nw, err);
          } else if (i < ib) {
            const uint32_t p = a.primes[i];
            const uint64_t m = a.magic[i];
            const uint32_t r = fma_mod ? mod_by_magic_fma(ktile, ks, p, m) : mod_barrett(ktile, p, m);
            const uint32_t pa = p / 30u, bi = (uint32_t)s_rb[p - 30u * pa];
            const uint2 st8 = reinterpret_cast<const uint2*>(s_step)[bi];  // the prime's 8 entries
#pragma unroll
            for (uint32_t o = 0; o < 8; ++o) {
              const uint32_t e = ((o < 4u ? st8.x : st8.y) >> (8u * (o & 3u))) & 0xFFu;
              const uint32_t delta = pa * w30(o) + (e & 31u);
              clear_progression(bm, delta >= r ? delta - r : delta + p - r, p, e >> 5, Lt, nw, err);
            }
          }
        }
      } else {
        // a lane per (prime, residue): a warp takes 4 consecutive primes, lane = 8*prime + residue
        const uint32_t o = (uint32_t)lane & 7u;
        const uint32_t wo = w30(o);
        const uint32_t groups = (ib - ia + 3u) >> 2;
        const uint32_t warp = (uint32_t)tid >> 5;
        for (uint32_t g = warp; g < groups; g += BLOCK / 32) {
          const uint32_t i = ia + 4u * g + ((uint32_t)lane >> 3);
          if (i < ib) {
            const uint32_t p = a.primes[i];
            const uint32_t r = mod_barrett(ktile, p, a.magic[i]);
            const uint32_t pa = p / 30u, bi = (uint32_t)s_rb[p - 30u * pa];
            const uint32_t e = s_step[bi * 8u + o];
            const uint32_t delta = pa * wo + (e & 31u);
            clear_progression(bm, delta >= r ? delta - r : delta + p - r, p, e >> 5, Lt, nw, err);
          }
        }
      }
      VOSS_PHASE(4)
      // large primes: walk the multiples of p across the tile's span of integers
      const uint64_t vbase = H.vbase;
      const uint32_t span = 30u * Lt;
      for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&H.c_ctr, 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base >= np - ib) break;
        const uint32_t i = ib + base + (uint32_t)lane;
        if (i < np) {
          const uint32_t p = a.primes[i];
          const uint64_t m = a.magic[i];
          const uint32_t r = fma_mod && p < (1u << 30) ? mod_by_magic_fma(vbase, vs, p, m) : mod_barrett(vbase, p, m);
          uint32_t d = r ? p - r : 0u;
          for (; d < span; d += p) {
            const uint32_t q = d / 30u;
            const int b = s_rb[d - 30u * q];
            if (b >= 0) clear_bit_word(bm, q >> 2, ~(1u << (((q & 3u) << 3) | (uint32_t)b)), nw, err);
          }
        }
      }
    }
    __syncthreads();
    VOSS_PHASE(5)

    // ---- 3. restore primes lying in the tile ---------------------------------------------
    {
      const uint64_t vbase = H.vbase, vlo = H.vlo, vhi = H.vhi, vend = vbase + 30ull * Lt;
      if (vbase < 32 && tid < 8) {
        const uint32_t sp[8] = {7, 11, 13, 17, 19, 23, 29, 31};
        const uint64_t p = sp[tid];
        if (p >= vlo && p < vhi && p >= vbase && p < vend) {
          const uint32_t off = (uint32_t)(p - vbase), k = off / 30u;
          atomicOr(bm + (k >> 2), 1u << (((k & 3u) << 3) | (uint32_t)s_rb[off - 30u * k]));
        }
      }
      for (uint32_t i = H.r0 + tid; i < H.r1; i += BLOCK) {
        const uint64_t p = a.primes[i];
        if (p >= vlo && p < vhi && p >= vbase && p < vend) {
          const uint32_t off = (uint32_t)(p - vbase), k = off / 30u;
          if ((k >> 2) < nw)
            atomicOr(bm + (k >> 2), 1u << (((k & 3u) << 3) | (uint32_t)s_rb[off - 30u * k]));
        }
      }
    }
    __syncthreads();
    VOSS_PHASE(6)

    // ---- 4. extract -----------------------------------------------------------------------
    const uint32_t c0 = (uint32_t)tid * C;
    const uint32_t cend = c0 < nw ? (c0 + C < nw ? c0 + C : nw) : c0;

    if (EMIT) {
      uint32_t pc = 0;
      for (uint32_t w = c0; w < cend; ++w) pc += __popc(bm[w]);
      uint32_t total;
      uint32_t rank = block_excl_sum<BLOCK>(pc, S, &total);
      const unsigned long long base = a.tile_offset[H.tile];
      const uint64_t vbase = H.vbase;
      for (uint32_t w = c0; w < cend; ++w) {
        uint32_t x = bm[w];
        while (x) {
          const uint32_t b = (uint32_t)__ffs(x) - 1u;
          x &= x - 1u;
          const unsigned long long idx = base + rank;
          if (idx < a.out_cap) a.out[idx] = vbase + 120ull * w + 30u * (b >> 3) + w30(b & 7u);
          ++rank;
        }
      }
      __syncthreads();
    } else {
      class_counts_by_word<BLOCK>(bm, nw, H.k28, H.k143, cnt, (uint32_t)lane, err);
      // pass 1: the primes of my chunk and its last prime
      uint32_t pc = 0;
      int32_t my_last = -1;
      const uint32_t cmid = c0 + (C >> 1) < cend ? c0 + (C >> 1) : cend;
#pragma unroll 4
      for (uint32_t w = c0; w < cmid; ++w) pc += (uint32_t)__popc(bm[w]);
      const uint32_t pc_half = pc;
#pragma unroll 4
      for (uint32_t w = cmid; w < cend; ++w) pc += (uint32_t)__popc(bm[w]);
      for (uint32_t w = cend; pc && w > c0;) {  // the chunk's last prime: its last non-zero word
        const uint32_t x = bm[--w];
        if (x) {
          my_last = (int32_t)(120u * w + s_pos[31u - (uint32_t)__clz(x)]);
          break;
        }
      }
      uint32_t tile_cnt;
      const uint32_t rank0 = block_excl_sum<BLOCK>(pc, S, &tile_cnt);
      int32_t tile_last;
      const int32_t before = block_excl_max<BLOCK>(my_last, S, &tile_last);
      s_rank[tid] = rank0;
      s_mid[tid] = (uint16_t)pc_half;
      s_before[tid] = before;
      __syncthreads();
      VOSS_PHASE(7)

      // pass 2: every thread walks the same number of the tile's primes in order (ranks
      // [ra, rb) of tile_cnt), so that the lanes of a warp run the same trip count.  The start
      // is the prime of rank ra: the chunk holding it is the last one whose first rank is <= ra.
      const uint32_t ra = (uint32_t)(((unsigned long long)tile_cnt * (uint32_t)tid) / BLOCK);
      const uint32_t rb = (uint32_t)(((unsigned long long)tile_cnt * ((uint32_t)tid + 1u)) / BLOCK);
      const uint32_t n_mine = rb - ra;
      uint32_t w = 0, x = 0;
      int32_t prev = -1;
      if (n_mine) {
        uint32_t lo = 0, hi = BLOCK;  // s_rank[lo] <= ra
        while (hi - lo > 1u) {
          const uint32_t mid = (lo + hi) >> 1;
          if (s_rank[mid] <= ra) lo = mid; else hi = mid;
        }
        uint32_t k = ra - s_rank[lo];
        w = lo * C;
        const uint32_t kh = s_mid[lo];
        if (k >= kh) {  // the start lies in the chunk's second half
          k -= kh;
          w += C >> 1;
        }
        x = bm[w];
        for (;;) {  // the word holding the start: it lies in chunk lo
          const uint32_t c = (uint32_t)__popc(x);
          if (k < c) break;
          k -= c;
          x = bm[++w];
        }
        if (k) {  // the primes of that word before mine: the last of them is my predecessor
          for (; k > 1u; --k) x &= x - 1u;
          prev = (int32_t)(120u * w + s_pos[(uint32_t)__ffs(x) - 1u]);
          x &= x - 1u;
        } else {  // mine is the word's first prime: the predecessor is in an earlier word
          prev = s_before[lo];
          for (uint32_t ww = w; ww > lo * C;) {
            const uint32_t y = bm[--ww];
            if (y) {
              prev = (int32_t)(120u * ww + s_pos[31u - (uint32_t)__clz(y)]);
              break;
            }
          }
        }
      }
      const uint32_t vb = H.vb;
      const uint32_t cthr = H.cthr;
      uint32_t mg = 0, mlo = 0;
      uint32_t o_prev = 0;  // wheel residue of the previous prime (modq counters: 8 * (g / 2) + o)
      if (prev >= 0) {
        const uint32_t kp = (uint32_t)prev / 30u;
        o_prev = (uint32_t)s_rb[(uint32_t)prev - 30u * kp];
      }
      uint32_t wpos = 120u * w;
      uint32_t it0 = 0;
      if (prev < 0 && n_mine) {
        // the tile's first prime: no predecessor in the tile (exactly one thread)
        while (x == 0u) {
          x = bm[++w];
          wpos += 120u;
        }
        const uint32_t b = (uint32_t)__ffs(x) - 1u;
        x &= x - 1u;
        const uint32_t pos = wpos + s_pos[b];
        H.first = pos;
        prev = (int32_t)pos;
        o_prev = b & 7u;
        it0 = 1;
      }
      uint32_t pv = (uint32_t)prev;
      // Instantiated twice: in a tile without a segment boundary (vb = kNone, nearly all of
      // them) the crossing test drops out of the loop.
      auto walk = [&](auto cross_tag) {
        constexpr bool kCross = decltype(cross_tag)::value;
        // unrolled by 4: one trip-count test per four primes (the count is known at entry)
#pragma unroll 4
        for (uint32_t it = it0; it < n_mine; ++it) {
          while (x == 0u) {  // the tile holds rb >= ra + it + 1 primes: w stays inside it
            x = bm[++w];
            wpos += 120u;
          }
          const uint32_t b = (uint32_t)__ffs(x) - 1u;
          x &= x - 1u;
          const uint32_t pos = wpos + s_pos[b];
          const uint32_t g = pos - pv;
          const bool crossing = kCross && (pv < vb) && (pos >= vb);
          const bool small = g < 100u && !crossing;
          if (small || g < 2u * kHistBins) {
            sm_add(cnt, small ? (uint32_t)kSmModq + 4u * g + o_prev : (uint32_t)kSmHist + (g >> 1), err);
          } else {
            atomicAdd(a.acc + (size_t)H.interval * kAccStride + kAccHistOver, 1ull);
            const uint32_t slot = atomicAdd(a.over_count, 1u);
            if (slot < a.over_cap) a.over[slot] = OverflowGap{H.interval, g};
            else atomicOr(err, kErrOverflowList);
          }
          mlo = g > mg ? pv : mlo;
          mg = g > mg ? g : mg;
          if (g >= cthr && !crossing) {
            const uint64_t v0 = H.vbase + pv;
            const double merit_d = (double)g / log((double)v0);
            if (a.large_min_gap || g >= 500u || merit_d >= 10.0) {
              const uint32_t slot = atomicAdd(a.large_count, 1u);
              if (slot < a.large_cap) {
                a.large[slot] = LargeGapDev{H.vbase + pos, (int32_t)g, (float)merit_d};
                a.large_iv[slot] = H.interval;
              }
            }
          }
          pv = pos;
          o_prev = b & 7u;
        }
      };
      if (vb == kNone) walk(std::false_type{});
      else walk(std::true_type{});
      const unsigned long long key =
          mg ? (((unsigned long long)mg << 32) | (unsigned long long)(0xFFFFFFFFu - mlo)) : 0ull;
      uint32_t tile_cnt2;
      unsigned long long tile_key;
      __syncthreads();  // H.first visible, scratch reuse
      VOSS_PHASE(8)
      block_reduce_tile<BLOCK>(n_mine, key, S, &tile_cnt2, &tile_key);
      (void)tile_cnt2;  // = tile_cnt
      if (tid == 0) {
        TilePartial P;
        P.first = tile_cnt ? H.first : kNone;
        P.last = tile_cnt ? (uint32_t)tile_last : kNone;
        P.count = tile_cnt;
        P.max_gap = (uint32_t)(tile_key >> 32);
        P.max_lo = tile_key ? 0xFFFFFFFFu - (uint32_t)(tile_key & 0xFFFFFFFFull) : 0u;
        P.bgap = 0;
        P.bgap_lo = 0;
        a.partials[H.tile] = P;
        St.count_total += tile_cnt;
        St.since_flush++;
      }
    }
    cur ^= 1u;
    __syncthreads();
    VOSS_PHASE(9)
  }
#ifdef VOSS_PHASE_TIMING
  if (threadIdx.x == 0)
    for (int k = 0; k < 10; ++k) atomicAdd(&g_phase_cycles[k], ph_acc[k]);
#endif
}

// Gap between the last prime of the previous non-empty tile and this tile's first prime.
__global__ void stitch_kernel(SieveArgs a) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= a.n_tiles) return;
  const TilePartial P = a.partials[t];
  if (P.count == 0) return;
  const uint32_t ivx = find_interval(a, t);
  const IntervalDev iv = a.iv[ivx];
  uint32_t tp = t;
  bool found = false;
  while (tp > iv.tile_begin) {
    --tp;
    if (a.partials[tp].count) {
      found = true;
      break;
    }
  }
  if (!found) return;
  const uint64_t kt = iv.k0 + 4ull * a.tile_words * (t - iv.tile_begin);
  const uint64_t kp = iv.k0 + 4ull * a.tile_words * (tp - iv.tile_begin);
  const uint64_t hi_p = 30ull * kt + P.first;
  const uint64_t lo_p = 30ull * kp + a.partials[tp].last;
  const uint64_t g = hi_p - lo_p;
  const bool crossing = iv.seg_k && ((lo_p / 30ull) / iv.seg_k != (hi_p / 30ull) / iv.seg_k);
  unsigned long long* acc = a.acc + (size_t)ivx * kAccStride;
  if (g < 100 && !crossing) {
    const uint32_t o_prev = (uint32_t)c_res_bit[lo_p % 30ull];
    atomicAdd(acc + kAccModq + o_prev * kModqBins + (g >> 1), 1ull);
  } else if (g < 2ull * kHistBins) {
    atomicAdd(acc + kAccHist + (g >> 1), 1ull);
  } else {
    atomicAdd(acc + kAccHistOver, 1ull);
    const uint32_t slot = atomicAdd(a.over_count, 1u);
    if (slot < a.over_cap) a.over[slot] = OverflowGap{ivx, (uint32_t)(g > 0xFFFFFFFFull ? 0xFFFFFFFFull : g)};
    else atomicOr(a.error, kErrOverflowList);
  }
  a.partials[t].bgap = (uint32_t)(g > 0xFFFFFFFFull ? 0xFFFFFFFFull : g);
  a.partials[t].bgap_lo = lo_p;
  const bool cand = a.large_min_gap ? (g >= a.large_min_gap) : (g > 100);
  if (a.want_large && cand && !crossing) {
    const double merit_d = (double)g / log((double)lo_p);
    if (a.large_min_gap || g >= 500 || merit_d >= 10.0) {
      const uint32_t slot = atomicAdd(a.large_count, 1u);
      if (slot < a.large_cap) {
        a.large[slot] = LargeGapDev{hi_p, (int32_t)g, (float)merit_d};
        a.large_iv[slot] = ivx;
      }
    }
  }
}

// One block per interval: first/last prime and the first maximal gap.
__global__ void reduce_kernel(SieveArgs a, IntervalOut* out) {
  const uint32_t ivx = blockIdx.x;
  if (ivx >= a.n_intervals) return;
  const IntervalDev iv = a.iv[ivx];
  __shared__ uint32_t s_first, s_last, s_gap;
  __shared__ unsigned long long s_lo;
  if (threadIdx.x == 0) {
    s_first = kNone;
    s_last = 0;
    s_gap = 0;
    s_lo = ~0ull;
  }
  __syncthreads();
  uint32_t my_first = kNone, my_last = 0, my_gap = 0;
  for (uint32_t i = threadIdx.x; i < iv.n_tiles; i += blockDim.x) {
    const TilePartial P = a.partials[iv.tile_begin + i];
    if (!P.count) continue;
    my_first = min(my_first, i);
    my_last = max(my_last, i + 1);
    my_gap = max(my_gap, max(P.max_gap, P.bgap));
  }
  atomicMin(&s_first, my_first);
  atomicMax(&s_last, my_last);
  atomicMax(&s_gap, my_gap);
  __syncthreads();
  const uint32_t G = s_gap;
  unsigned long long my_lo = ~0ull;
  if (G) {
    for (uint32_t i = threadIdx.x; i < iv.n_tiles; i += blockDim.x) {
      const TilePartial P = a.partials[iv.tile_begin + i];
      if (!P.count) continue;
      const uint64_t vt = 30ull * (iv.k0 + 4ull * a.tile_words * i);
      if (P.max_gap == G) my_lo = min(my_lo, (unsigned long long)(vt + P.max_lo));
      if (P.bgap == G) my_lo = min(my_lo, (unsigned long long)P.bgap_lo);
    }
  }
  atomicMin(&s_lo, my_lo);
  __syncthreads();
  if (threadIdx.x == 0) {
    IntervalOut o;
    if (s_first == kNone) {
      o.first = o.last = 0;
    } else {
      const TilePartial F = a.partials[iv.tile_begin + s_first];
      const TilePartial L = a.partials[iv.tile_begin + s_last - 1];
      o.first = 30ull * (iv.k0 + 4ull * a.tile_words * s_first) + F.first;
      o.last = 30ull * (iv.k0 + 4ull * a.tile_words * (s_last - 1)) + L.last;
    }
    o.max_gap = G;
    o.max_gap_lo = G ? s_lo : 0;
    out[ivx] = o;
  }
}

// One block per interval: fold the accumulators into voss_interval_stats on the device, so
// that only the result (not the raw counters) crosses to the host.  lo/hi and the primes
// 2, 3, 5 are filled in on the host.
__global__ void interval_finalize_kernel(SieveArgs a, const IntervalOut* io, voss_interval_stats* out,
                                         const uint32_t* out_index) {
  const uint32_t ivx = blockIdx.x;
  if (ivx >= a.n_intervals) return;
  const unsigned long long* A = a.acc + (size_t)ivx * kAccStride;
  voss_interval_stats* s = out + (out_index ? out_index[ivx] : ivx);
  for (uint32_t b = threadIdx.x; b < (uint32_t)VOSS_IHIST; b += blockDim.x) {
    unsigned long long v = 0;
    if (b > 0) {
      v = A[kAccHist + b];
      if (b < (uint32_t)kModqBins)
        for (uint32_t o = 0; o < 8; ++o) v += A[kAccModq + o * kModqBins + b];
    }
    s->gap_hist[b] = v;
  }
  if (threadIdx.x == 0) {
    s->lo = 0;
    s->hi = 0;
    s->prime_count = A[kAccCount];
    s->first_prime = io[ivx].first;
    s->last_prime = io[ivx].last;
    s->max_gap = io[ivx].max_gap;
    s->max_gap_lo = io[ivx].max_gap_lo;
    s->gap_overflow = A[kAccHistOver];
  }
}

int launch_interval_finalize(const SieveArgs& a, const IntervalOut* io, voss_interval_stats* out,
                             const uint32_t* out_index, void* stream) {
  if (a.n_intervals == 0) return 0;
  interval_finalize_kernel<<<a.n_intervals, 256, 0, (cudaStream_t)stream>>>(a, io, out, out_index);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Large-prime pre-pass (bucket-free): each thread takes primes p >= 8 * tile bytes in turn and,
// for every interval of the launch that p can reach (intervals sorted by isqrt(hi - 1),
// descending, staged in shared memory), walks p's multiples across the interval and clears
// them in the launch's large-prime bitmap with global atomics.  The prime table is read once
// per launch instead of once per tile, which is what bounds high intervals (at 1e18 the table
// is 610 MB).  The tile kernel ANDs this bitmap into its fill and skips these primes.
constexpr int kScatterChunk = 960;  // 45 KB of interval descriptors per block

__global__ void __launch_bounds__(512) scatter_large_kernel(const uint32_t* __restrict__ primes,
                                                            const uint64_t* __restrict__ magic, uint32_t j0,
                                                            uint32_t j1, const IntervalScatter* __restrict__ iv,
                                                            uint32_t n_iv, uint32_t* __restrict__ gbm) {
  __shared__ IntervalScatter s_iv[kScatterChunk];
  __shared__ int8_t s_rb[32];
  __shared__ uint8_t s_wstart[240];
  __shared__ uint2 s_wstep[64];
  if (threadIdx.x < 32) s_rb[threadIdx.x] = c_res_bit[threadIdx.x];
  if (threadIdx.x < 240) s_wstart[threadIdx.x] = c_walk_start[threadIdx.x];
  if (threadIdx.x < 64) s_wstep[threadIdx.x] = c_walk_step[threadIdx.x];
  for (uint32_t i = threadIdx.x; i < n_iv; i += blockDim.x) s_iv[i] = iv[i];
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t j = j0 + blockIdx.x * blockDim.x + threadIdx.x; j < j1; j += stride) {
    const uint32_t p = primes[j];  // >= 8 tile spans >= 2^11 (mod_by_estimate's range)
    const double inv = __drcp_rn((double)p);
    const uint32_t pa = p / 30u, bi = (uint32_t)s_rb[p - 30u * pa];
    const uint2* row = s_wstep + bi * 8u;
    const bool narrow = p < (1u << 30);
    // intervals are sorted by sqrt_hi, descending: p reaches the first n_reach of them
    uint32_t lo = 0, hi = n_iv;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (s_iv[mid].sqrt_hi >= p) lo = mid + 1; else hi = mid;
    }
    const uint32_t n_reach = lo;
#pragma unroll 4
    for (uint32_t s = 0; s < n_reach; ++s) {
      // one 16-byte load per pair: (vbase_d, vbase_lo, span32)
      const uint4 h = *reinterpret_cast<const uint4*>(&s_iv[s]);
      const double vd = __hiloint2double((int)h.y, (int)h.x);
      // q = vbase / p rounded to an integer: adding 2^52 in the same rounding leaves the
      // integer in the low mantissa bits (q < 2^52), so no conversion instruction is needed
      const double qd = __fma_rn(vd, inv, 4503599627370496.0);
      uint32_t d;  // first multiple of p, offset from vbase
      if (narrow) {  // 32-bit arithmetic: r = vbase - q p as int32 in (-p, 2p)
        uint32_t r = h.z - (uint32_t)__double2loint(qd) * p;
        r += (int32_t)r < 0 ? p : 0u;
        r -= r >= p ? p : 0u;
        d = r ? p - r : 0u;
      } else {
        const unsigned long long q = (unsigned long long)(__double_as_longlong(qd) - 0x4330000000000000ll);
        int64_t rr = (int64_t)(s_iv[s].vbase - q * (uint64_t)p);
        rr += rr < 0 ? (int64_t)p : 0;
        rr -= rr >= (int64_t)p ? (int64_t)p : 0;
        d = rr ? p - (uint32_t)rr : 0u;
      }
      if (d >= h.w) continue;                      // none in the interval
      const uint2 sp_lt = make_uint2(h.w, s_iv[s].lt32);
      const IntervalScatter& I = s_iv[s];
      if (sp_lt.y) {
        // wheel walk over the multiples p*m with gcd(m, 30) = 1 (vbase is a multiple of 30)
        const uint32_t st = s_wstart[bi * 30u + (d - 30u * (d / 30u))];
        const uint64_t off = (uint64_t)d + (uint64_t)(st & 7u) * p;
        if (off >= I.span) continue;
        uint32_t byte = (uint32_t)(off / 30ull), w = st >> 3;
        const uint32_t lt = sp_lt.y;
        uint32_t* g = gbm + I.gword;
        while (byte < lt) {
          const uint2 e = row[w];
          atomicAnd(g + (byte >> 2), __funnelshift_l(e.x, e.x, byte << 3));
          byte += pa * (e.y & 0xFFFFu) + (e.y >> 16);
          w = (w + 1u) & 7u;
        }
      } else {
        for (uint64_t dd = d; dd < I.span; dd += p) {
          const uint64_t q64 = dd / 30ull;
          const int b = s_rb[(uint32_t)(dd - 30ull * q64)];
          if (b >= 0) atomicAnd(gbm + I.gword + (q64 >> 2), ~(1u << ((((uint32_t)q64 & 3u) << 3) | (uint32_t)b)));
        }
      }
    }
  }
}

int launch_scatter_large(const uint32_t* primes, const uint64_t* magic, uint32_t j0, uint32_t j1,
                         const IntervalScatter* iv, uint32_t n_iv, uint32_t* gbm, int sm_count, void* stream) {
  if (ensure_tables()) return -1;
  if (j1 <= j0 || n_iv == 0) return 0;
  const uint32_t per = 512u;
  const uint64_t want = ((uint64_t)(j1 - j0) + per - 1) / per;
  const int grid = (int)(want < (uint64_t)sm_count * 4 ? want : (uint64_t)sm_count * 4);
  for (uint32_t off = 0; off < n_iv; off += kScatterChunk) {
    const uint32_t n = n_iv - off < (uint32_t)kScatterChunk ? n_iv - off : (uint32_t)kScatterChunk;
    scatter_large_kernel<<<grid, per, 0, (cudaStream_t)stream>>>(primes, magic, j0, j1, iv + off, n, gbm);
  }
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---- shared-memory RMW probe ------------------------------------------------------------
constexpr int kProbeWords = 8192;
constexpr int kProbeIters = 4096;

__global__ void __launch_bounds__(1024) smem_rmw_probe_kernel(uint32_t* sink) {
  __shared__ uint32_t s[kProbeWords];
  for (int i = threadIdx.x; i < kProbeWords; i += blockDim.x) s[i] = 0xFFFFFFFFu;
  __syncthreads();
  uint32_t idx = threadIdx.x;
#pragma unroll 8
  for (int it = 0; it < kProbeIters; ++it) {
    atomicAnd(&s[idx & (kProbeWords - 1)], ~(1u << (it & 31)));
    idx += 1024u;
  }
  __syncthreads();
  if (threadIdx.x == 0) sink[blockIdx.x] = s[blockIdx.x & (kProbeWords - 1)];
}

// ---- host side ------------------------------------------------------------------------------
#ifdef VOSS_PHASE_TIMING
int read_phase_cycles(unsigned long long* out, int n, bool reset) {
  unsigned long long h[16];
  if (cudaMemcpyFromSymbol(h, g_phase_cycles, sizeof(h)) != cudaSuccess) return -1;
  for (int i = 0; i < n && i < 16; ++i) out[i] = h[i];
  if (reset) {
    unsigned long long z[16] = {0};
    if (cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z)) != cudaSuccess) return -1;
  }
  return 0;
}
#endif
static const int kW30h[8] = {1, 7, 11, 13, 17, 19, 23, 29};

static int ensure_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
  const uint64_t bit = 1ull << dev;
  if (g_tables_ready.load() & bit) return 0;
  uint8_t step[64];
  int8_t rb[32];
  for (int r = 0; r < 32; ++r) rb[r] = -1;
  for (int i = 0; i < 8; ++i) rb[kW30h[i]] = (int8_t)i;
  for (int bi = 0; bi < 8; ++bi)
    for (int o = 0; o < 8; ++o) {
      const int bw = kW30h[bi] * kW30h[o];
      step[bi * 8 + o] = (uint8_t)((bw / 30) | (rb[bw % 30] << 5));
    }
  uint8_t wstart[240];
  uint2 wstep[64];
  uint32_t wpk[16] = {0};
  for (int bi = 0; bi < 8; ++bi) {
    int pinv = 1;
    while ((kW30h[bi] * pinv) % 30 != 1) ++pinv;
    for (int t = 0; t < 30; ++t) {
      const int u = (t * pinv) % 30;
      int adv = 0;
      while (rb[(u + adv) % 30] < 0) ++adv;
      wstart[bi * 30 + t] = (uint8_t)(adv | (rb[(u + adv) % 30] << 3));
    }
    for (int j = 0; j < 8; ++j) {
      const int w = kW30h[bi];
      const int d0 = (w * kW30h[j]) / 30;
      const int gap = (j < 7 ? kW30h[j + 1] : 31) - kW30h[j];
      const int corr = j < 7 ? (w * kW30h[j + 1]) / 30 - d0 : w + 0 - d0;  // j = 7: next m is 30(c+1) + 1
      wstep[bi * 8 + j] = make_uint2(~(1u << rb[(w * kW30h[j]) % 30]), (uint32_t)gap | ((uint32_t)corr << 16));
      wpk[bi] |= (uint32_t)corr << (4 * j);
      wpk[8 + bi] |= (uint32_t)rb[(w * kW30h[j]) % 30] << (4 * j);
    }
  }
  if (cudaMemcpyToSymbol(c_walk_start, wstart, sizeof(wstart)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_walk_step, wstep, sizeof(wstep)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_walk_pk, wpk, sizeof(wpk)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_wheel_step, step, sizeof(step)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_res_bit, rb, sizeof(rb)) != cudaSuccess) return -1;
  g_tables_ready.fetch_or(bit);
  return 0;
}

void build_presieve_tables(uint32_t* out) {
  static const uint32_t groups[kPreGroups][3] = {{7, 11, 13}, {17, 19, 0}, {23, 29, 0}, {31, 0, 0}};
  for (int g = 0; g < kPreGroups; ++g) {
    const uint32_t P = kPreMod[g];
    for (uint32_t j = 0; j < P; ++j) {
      uint32_t m = 0xFFFFFFFFu;
      for (uint32_t jb = 0; jb < 4; ++jb)
        for (uint32_t o = 0; o < 8; ++o) {
          const uint64_t k = 4ull * j + jb;  // byte index modulo P
          for (int q = 0; q < 3 && groups[g][q]; ++q) {
            const uint32_t p = groups[g][q];
            if ((30ull * k + kW30h[o]) % p == 0) m &= ~(1u << (8 * jb + o));
          }
        }
      out[kPreOff[g] + j] = m;
    }
  }
}

size_t sieve_smem_bytes(uint32_t tile_words) {
  return (size_t)(tile_words + kPreWords + kSmCounters) * sizeof(uint32_t);
}

template <int BLOCK, bool EMIT>
static int set_attrs(size_t smem) {
  auto fn = sieve_tiles_kernel<BLOCK, EMIT>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  return 0;
}

int sieve_kernel_attrs(int block, size_t smem, int* max_ctas_per_sm) {
  if (ensure_tables()) return -1;
  int rc = 0, n = 0;
  if (block == 512) {
    rc |= set_attrs<512, false>(smem) | set_attrs<512, true>(smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sieve_tiles_kernel<512, false>, 512, smem) != cudaSuccess) rc = -1;
  } else if (block == 1024) {
    rc |= set_attrs<1024, false>(smem) | set_attrs<1024, true>(smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, sieve_tiles_kernel<1024, false>, 1024, smem) != cudaSuccess) rc = -1;
  } else {
    return -1;
  }
  if (max_ctas_per_sm) *max_ctas_per_sm = n;
  return rc;
}

int launch_sieve_stats(const SieveArgs& a, int grid, int block, size_t smem, void* stream) {
  if (ensure_tables()) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  if (block == 512) sieve_tiles_kernel<512, false><<<grid, 512, smem, s>>>(a);
  else if (block == 1024) sieve_tiles_kernel<1024, false><<<grid, 1024, smem, s>>>(a);
  else return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_sieve_emit(const SieveArgs& a, int grid, int block, size_t smem, void* stream) {
  if (ensure_tables()) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  if (block == 512) sieve_tiles_kernel<512, true><<<grid, 512, smem, s>>>(a);
  else if (block == 1024) sieve_tiles_kernel<1024, true><<<grid, 1024, smem, s>>>(a);
  else return -1;
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_stitch(const SieveArgs& a, void* stream) {
  if (a.n_tiles == 0) return 0;
  const int blk = 256;
  stitch_kernel<<<(a.n_tiles + blk - 1) / blk, blk, 0, (cudaStream_t)stream>>>(a);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_reduce(const SieveArgs& a, IntervalOut* out, void* stream) {
  if (a.n_intervals == 0) return 0;
  reduce_kernel<<<a.n_intervals, 256, 0, (cudaStream_t)stream>>>(a, out);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int probe_smem_rmw(int sm_count, void* stream, float* ms, double* bytes) {
  cudaStream_t s = (cudaStream_t)stream;
  const int grid = sm_count * 2;
  uint32_t* sink = nullptr;
  if (cudaMalloc(&sink, grid * sizeof(uint32_t)) != cudaSuccess) return -1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  smem_rmw_probe_kernel<<<grid, 1024, 0, s>>>(sink);  // warm-up
  cudaEventRecord(e0, s);
  const int reps = 5;
  for (int r = 0; r < reps; ++r) smem_rmw_probe_kernel<<<grid, 1024, 0, s>>>(sink);
  cudaEventRecord(e1, s);
  cudaError_t st = cudaEventSynchronize(e1);
  float t = 0;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (st != cudaSuccess) return -1;
  *ms = t / reps;
  *bytes = (double)grid * 1024.0 * kProbeIters * 8.0;
  return 0;
}

}  // namespace voss

// mr_kernels.cu — deterministic Miller-Rabin and gap proofs on sm_100a.
//
// Result-for-result equal to the reference verifier src/verify_cpp.cpp:
//   is_prime_u64 (:38-57): n < 2 -> composite; for each base B in {2,...,37}: n == B -> prime,
//   B | n -> composite; then the strong-probable-prime test to every base.
//   verify_gap (:59-93): both ends prime, then every interior integer must be marked by the
//   interval sieve (evens, then odd multiples of the odd base primes q <= isqrt(p_after)).
//
// Arithmetic: 64-bit Montgomery multiplication with R = 2^64 (mul.lo/mul.hi on the integer
// pipe, no 128-bit division); the reference's u128 '%' (verify_cpp.cpp:24) is not used.
// Base 2 is special-cased: its square-and-multiply multiplies by 2 with a modular addition.
// Work is split in two kernels so that warps stay full: mr_sieve_kernel resolves every
// candidate that trial division or base 2 decides (nearly all composites) and appends the rest
// to a work list; mr_finish_kernel runs the remaining bases on that list, as many as the size
// of n requires for an exact verdict (bases_needed: 6, 7, 9 or all 12), so its results equal
// the reference's twelve-base test for every 64-bit n.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "voss.h"

#include "voss_internal.h"

namespace voss {

__constant__ uint64_t c_base_inv[12];  // B^-1 mod 2^64 (odd B), for the divisibility test
__constant__ uint64_t c_base_lim[12];  // floor((2^64-1)/B)

// Constant memory is per device: the tables are uploaded once for each device ordinal.
static std::atomic<uint64_t> g_mr_ready{0};
static const uint64_t kBases[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};

struct Mont {
  uint64_t n, ninv, one, mone;
};

__device__ __forceinline__ uint64_t mont_mul(uint64_t a, uint64_t b, const Mont& M) {
  const uint64_t lo = a * b;
  const uint64_t hi = __umul64hi(a, b);
  const uint64_t m = lo * M.ninv;
  const uint64_t mh = __umul64hi(m, M.n);
  // (a*b + m*n) / 2^64 = hi + mh + carry, carry = (lo != 0) because lo + (m*n mod 2^64) = 0 mod 2^64
  const uint64_t t = hi + mh;
  const bool c1 = t < hi;
  const uint64_t t2 = t + (lo != 0 ? 1ull : 0ull);
  const bool c2 = t2 < t;
  return (c1 || c2 || t2 >= M.n) ? t2 - M.n : t2;
}

// mont_mul for n < 2^63: hi + mh < 2n < 2^64 and the low-half carry keeps it <= 2n, so no
// 64-bit overflow checks are needed.
__device__ __forceinline__ uint64_t mont_mul_small(uint64_t a, uint64_t b, const Mont& M) {
  const uint64_t lo = a * b;
  const uint64_t hi = __umul64hi(a, b);
  const uint64_t m = lo * M.ninv;
  const uint64_t t = hi + __umul64hi(m, M.n) + (lo != 0 ? 1ull : 0ull);
  return t >= M.n ? t - M.n : t;
}

__device__ __forceinline__ uint64_t mod_add(uint64_t a, uint64_t b, uint64_t n) {
  const uint64_t s = a + b;
  return (s < a || s >= n) ? s - n : s;
}

// 2^64 mod n for odd n > 1.  For n >= 2^32 the quotient q* = floor(2^64 / n), 1 <= q* < 2^32,
// is estimated in double precision (relative error < 2^-51, so the estimate is off by at most 1)
// and lowered by one, but not below 1: then q* - 2 <= q <= q* and q >= 1, so 2^64 - q n is below
// 2^64, lies in [0, 3n), and at most two subtractions finish it.  Smaller n take the 64-bit
// integer remainder.
__device__ __forceinline__ uint64_t two64_mod(uint64_t n) {
  if (n < (1ull << 32)) return (0ull - n) % n;
  uint64_t q = (uint64_t)(18446744073709551616.0 / (double)n);
  q = q > 1 ? q - 1 : 1;
  uint64_t r = 0ull - q * n;  // 2^64 - q n
  if (r >= n) r -= n;
  if (r >= n) r -= n;
  return r;
}

__device__ __forceinline__ Mont mont_setup(uint64_t n) {
  Mont M;
  M.n = n;
  uint64_t x = n;  // inverse of n mod 2^3
#pragma unroll
  for (int i = 0; i < 5; ++i) x *= 2ull - n * x;
  M.ninv = 0ull - x;
  M.one = two64_mod(n);  // R mod n
  M.mone = n - M.one;
  return M;
}

// Trial phase of is_prime_u64: 1 = prime, 0 = composite, -1 = undecided.
__device__ __forceinline__ int trial_phase(uint64_t n) {
  if (n < 2) return 0;
  if (n == 2) return 1;
  if ((n & 1ull) == 0) return 0;
#pragma unroll
  for (int i = 1; i < 12; ++i) {
    const uint64_t B = i == 1 ? 3 : i == 2 ? 5 : i == 3 ? 7 : i == 4 ? 11 : i == 5 ? 13 : i == 6 ? 17
                     : i == 7 ? 19 : i == 8 ? 23 : i == 9 ? 29 : i == 10 ? 31 : 37;
    if (n == B) return 1;
    if (n * c_base_inv[i] <= c_base_lim[i]) return 0;
  }
  return -1;
}

// How many of the bases 2, 3, 5, ..., 37 (in this order) decide primality exactly for n.  The
// smallest strong pseudoprimes to the first k prime bases are 3,474,749,660,383 (k = 6),
// 341,550,071,728,321 (k = 7, 8) and 3,825,123,056,546,413,051 (k = 9..11) (Jaeschke 1993; OEIS
// A014233); below them the first 6, 7 or 9 bases already give the same verdict as all twelve,
// which remain exact for every n < 2^64.
__device__ __forceinline__ int bases_needed(uint64_t n) {
  return n < 3474749660383ull ? 6 : (n < 341550071728321ull ? 7 : (n < 3825123056546413051ull ? 9 : 12));
}
constexpr uint64_t kSmallMr = 3474749660383ull;  // survivors below go to the front work list

// Strong probable-prime test of odd n > 37 to the base whose Montgomery form is am.
__device__ __forceinline__ bool sprp(const Mont& M, uint64_t am, uint64_t d, int r) {
  uint64_t x = M.one;
  const int top = 63 - __clzll(d);
  for (int b = top; b >= 0; --b) {
    x = mont_mul(x, x, M);
    if ((d >> b) & 1ull) x = mont_mul(x, am, M);
  }
  if (x == M.one || x == M.mone) return true;
  for (int j = 0; j < r - 1; ++j) {
    x = mont_mul(x, x, M);
    if (x == M.mone) return true;
  }
  return false;
}

__device__ __forceinline__ bool sprp2(const Mont& M, uint64_t d, int r) {
  uint64_t x = M.one;
  const int top = 63 - __clzll(d);
  for (int b = top; b >= 0; --b) {
    x = mont_mul(x, x, M);
    if ((d >> b) & 1ull) x = mod_add(x, x, M.n);
  }
  if (x == M.one || x == M.mone) return true;
  for (int j = 0; j < r - 1; ++j) {
    x = mont_mul(x, x, M);
    if (x == M.mone) return true;
  }
  return false;
}

// Bases 3..37 (Montgomery forms built from R by modular additions).
__device__ __forceinline__ bool sprp_rest(const Mont& M, uint64_t d, int r) {
  const uint64_t n = M.n;
  const uint64_t r1 = M.one, r2 = mod_add(r1, r1, n), r4 = mod_add(r2, r2, n), r6 = mod_add(r4, r2, n);
  uint64_t a = mod_add(r2, r1, n);  // 3R
  // gaps between consecutive bases 3,5,7,11,13,17,19,23,29,31,37
  const int steps[10] = {2, 2, 4, 2, 4, 2, 4, 6, 2, 6};
  if (!sprp(M, a, d, r)) return false;
#pragma unroll
  for (int i = 0; i < 10; ++i) {
    const int s = steps[i];
    a = mod_add(a, s == 2 ? r2 : (s == 4 ? r4 : r6), n);
    if (!sprp(M, a, d, r)) return false;
  }
  return true;
}

__device__ bool is_prime_u64_dev(uint64_t n) {
  const int t = trial_phase(n);
  if (t >= 0) return t == 1;
  const Mont M = mont_setup(n);
  uint64_t d = n - 1;
  const int r = __ffsll((long long)d) - 1;
  d >>= r;
  if (!sprp2(M, d, r)) return false;
  return sprp_rest(M, d, r);
}

// Warp-uniform strong probable-prime test: every lane runs the same number of squarings and
// multiplications (the warp's longest exponent and largest r) and keeps its verdict in a flag.
// Early exits inside these loops let the lanes of a warp drift apart and never reconverge
// (measured: 2.8 active lanes per instruction); uniform loops keep all 32 lanes in step.
// kSmallN: every lane's n < 2^63 (mont_mul_small).
template <bool kSmallN = false>
__device__ __forceinline__ bool sprp_uniform(const Mont& M, uint64_t am, uint64_t d, int r, int top_w, int r_w,
                                             bool base2) {
  uint64_t x = M.one;
  for (int b = top_w; b >= 0; --b) {
    x = kSmallN ? mont_mul_small(x, x, M) : mont_mul(x, x, M);
    const uint64_t y = base2 ? mod_add(x, x, M.n) : (kSmallN ? mont_mul_small(x, am, M) : mont_mul(x, am, M));
    x = ((d >> b) & 1ull) ? y : x;
  }
  bool ok = (x == M.one) | (x == M.mone);
  for (int j = 0; j < r_w - 1; ++j) {
    x = kSmallN ? mont_mul_small(x, x, M) : mont_mul(x, x, M);
    ok |= (j < r - 1) & (x == M.mone);
  }
  return ok;
}

// sprp_uniform for a base whose products are real multiplications, with 2-bit exponent digits:
// x <- x^4 * a^digit for each digit of d from the top, a^0 = R, a, a^2, a^3 precomputed and
// picked by selects (no memory).  A base then costs about 1.5 products per bit of d instead of
// the 2 of the bitwise loop, which must multiply at every bit because some lane's bit is set.
template <bool kSmallN>
__device__ __forceinline__ bool sprp_uniform_w2(const Mont& M, uint64_t am, uint64_t d, int r, int top_w, int r_w) {
  const uint64_t a2 = kSmallN ? mont_mul_small(am, am, M) : mont_mul(am, am, M);
  const uint64_t a3 = kSmallN ? mont_mul_small(a2, am, M) : mont_mul(a2, am, M);
  // an odd number of bits (top_w even) starts with the single top bit, then bit pairs (b, b - 1)
  uint64_t x;
  int b;
  if ((top_w & 1) == 0) {
    x = ((d >> top_w) & 1ull) ? am : M.one;
    b = top_w - 1;
  } else {
    const uint32_t g = (uint32_t)(d >> (top_w - 1)) & 3u;
    x = g == 0u ? M.one : (g == 1u ? am : (g == 2u ? a2 : a3));
    b = top_w - 2;
  }
  for (; b >= 1; b -= 2) {
    x = kSmallN ? mont_mul_small(x, x, M) : mont_mul(x, x, M);
    x = kSmallN ? mont_mul_small(x, x, M) : mont_mul(x, x, M);
    const uint32_t g = (uint32_t)(d >> (b - 1)) & 3u;
    const uint64_t t = g == 0u ? M.one : (g == 1u ? am : (g == 2u ? a2 : a3));
    x = kSmallN ? mont_mul_small(x, t, M) : mont_mul(x, t, M);
  }
  bool ok = (x == M.one) | (x == M.mone);
  for (int j = 0; j < r_w - 1; ++j) {
    x = kSmallN ? mont_mul_small(x, x, M) : mont_mul(x, x, M);
    ok |= (j < r - 1) & (x == M.mone);
  }
  return ok;
}

// Bases 3, 5, 7, ... of mr_finish_kernel for one warp: each lane stops after bases_needed(n)
// bases or its first failure; the warp stops when no lane wants another base.
template <bool kSmallN>
__device__ __forceinline__ bool sprp_bases_3_on(const Mont& M, uint64_t d, int r, int top_w, int r_w, int need) {
  const uint64_t n_ = M.n;
  const uint64_t r1 = M.one, r2 = mod_add(r1, r1, n_), r4 = mod_add(r2, r2, n_), r6 = mod_add(r4, r2, n_);
  uint64_t a = mod_add(r2, r1, n_);  // 3R: bases 3,5,7,11,13,17,19,23,29,31,37 by their gaps
  bool prime = sprp_uniform_w2<kSmallN>(M, a, d, r, top_w, r_w);
#pragma unroll 1
  for (int s = 0; s < 10; ++s) {
    // base index s + 2 (5, 7, 11, ...): still wanted by a lane that is prime so far and needs it
    const bool want = prime && (s + 2 < need);
    if (!__any_sync(0xFFFFFFFFu, want)) break;
    const int step = (0x6264242422ull >> (4 * s)) & 0xF;  // 2,2,4,2,4,2,4,6,2,6
    a = mod_add(a, step == 2 ? r2 : (step == 4 ? r4 : r6), n_);
    const bool pass = sprp_uniform_w2<kSmallN>(M, a, d, r, top_w, r_w);
    prime = want ? pass : prime;
  }
  return prime;
}

// Trial division for every candidate (a lane per candidate), then base 2 for the undecided ones:
// those wait in the warp's shared-memory queues, one for n below 3,474,749,660,383 (exponents of
// at most 42 bits, six bases needed) and one for the rest, and each time a queue holds 32 they are
// tested together with warp-uniform loops (sprp_uniform), a lane each.  Lanes whose candidate
// trial division decides, and short exponents beside long ones, would otherwise leave most of the
// warp idle (13 of 32 lanes active per instruction when each lane ran its own test).  Base-2
// survivors go to the work list: the small ones from the front, the others from the back, so that
// the warps of mr_finish_kernel mostly share one base count.
constexpr int kSieveBlock = 256;
constexpr int kMrQueue = 64;  // per warp and size class: at most 31 waiting + 32 arriving

__device__ __forceinline__ void mr_base2_drain(const uint64_t* __restrict__ cand, uint8_t* __restrict__ out,
                                               uint32_t* __restrict__ work, uint32_t* __restrict__ nwork,
                                               uint64_t count, uint32_t* q, uint32_t& nq, bool small_class,
                                               uint32_t lane) {
  __syncwarp();
  const uint32_t take = nq < 32u ? nq : 32u;
  const bool live = lane < take;
  uint32_t i = live ? q[lane] : 0u;
  __syncwarp();
  if (lane + 32u < nq) q[lane] = q[lane + 32u];
  nq -= take;
  __syncwarp();
  const uint32_t i0 = __shfl_sync(0xFFFFFFFFu, i, 0);  // idle lanes shadow lane 0
  if (!live) i = i0;
  const uint64_t n = cand[i];
  const Mont M = mont_setup(n);
  uint64_t d = n - 1;
  const int r = __ffsll((long long)d) - 1;
  d >>= r;
  const int top_w = __reduce_max_sync(0xFFFFFFFFu, (unsigned)(63 - __clzll(d)));
  const int r_w = __reduce_max_sync(0xFFFFFFFFu, (unsigned)r);
  const bool ok = __all_sync(0xFFFFFFFFu, n < (1ull << 63)) ? sprp_uniform<true>(M, 0, d, r, top_w, r_w, true)
                                                           : sprp_uniform<false>(M, 0, d, r, top_w, r_w, true);
  if (live && !ok) out[i] = 0;
  const bool keep = live && ok;
  const unsigned mk = __ballot_sync(0xFFFFFFFFu, keep);
  if (mk) {
    uint32_t at = 0;
    if (lane == 0) at = atomicAdd(nwork + (small_class ? 0 : 1), (uint32_t)__popc(mk));
    at = __shfl_sync(0xFFFFFFFFu, at, 0) + (uint32_t)__popc(mk & ((1u << lane) - 1u));
    if (keep) {
      if (small_class) work[at] = i;
      else work[count - 1 - at] = i;
    }
  }
}

__global__ void __launch_bounds__(kSieveBlock) mr_sieve_kernel(const uint64_t* __restrict__ cand, uint64_t count,
                                                              uint8_t* __restrict__ out, uint32_t* __restrict__ work,
                                                              uint32_t* __restrict__ nwork) {
  __shared__ uint32_t s_q[kSieveBlock / 32][2][kMrQueue];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t* qs = s_q[warp][0];
  uint32_t* ql = s_q[warp][1];
  uint32_t ns = 0, nl = 0;  // warp-uniform queue lengths
  const unsigned below = (1u << lane) - 1u;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + 32u * warp; base < count; base += stride) {
    const uint64_t i = base + lane;
    bool und = false, small = false;
    if (i < count) {
      const uint64_t n = cand[i];
      const int t = trial_phase(n);
      if (t >= 0) out[i] = (uint8_t)t;
      else {
        und = true;
        small = n < kSmallMr;
      }
    }
    const unsigned ms = __ballot_sync(0xFFFFFFFFu, und && small);
    const unsigned ml = __ballot_sync(0xFFFFFFFFu, und && !small);
    if (und && small) qs[ns + __popc(ms & below)] = (uint32_t)i;
    if (und && !small) ql[nl + __popc(ml & below)] = (uint32_t)i;
    ns += __popc(ms);
    nl += __popc(ml);
    if (ns >= 32u) mr_base2_drain(cand, out, work, nwork, count, qs, ns, true, lane);
    if (nl >= 32u) mr_base2_drain(cand, out, work, nwork, count, ql, nl, false, lane);
  }
  if (ns) mr_base2_drain(cand, out, work, nwork, count, qs, ns, true, lane);
  if (nl) mr_base2_drain(cand, out, work, nwork, count, ql, nl, false, lane);
}

// `work` holds candidate indices (< 2^32: the entry points take fewer than 2^32 candidates per call):
// nwork[0] of them at the front, nwork[1] at the back (work[count - 1], work[count - 2], ...).
__global__ void mr_finish_kernel(const uint64_t* __restrict__ cand, uint8_t* __restrict__ out,
                                 const uint32_t* __restrict__ work, const uint32_t* __restrict__ nwork,
                                 uint32_t count) {
  const uint32_t na = nwork[0];
  const uint32_t nw = na + nwork[1];
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = warp0 * 32u; base < nw; base += nwarps * 32u) {  // warp-uniform loop
    const uint32_t k = base + lane;
    const bool live = k < nw;
    const uint32_t i = live ? work[k < na ? k : count - 1 - (k - na)] : 0u;
    uint64_t n = live ? cand[i] : 0ull;
    const uint64_t n0 = __shfl_sync(0xFFFFFFFFu, n, 0);  // idle lanes shadow lane 0
    if (!live) n = n0;
    const Mont M = mont_setup(n);
    uint64_t d = n - 1;
    const int r = __ffsll((long long)d) - 1;
    d >>= r;
    const int top = 63 - __clzll(d);
    const int top_w = __reduce_max_sync(0xFFFFFFFFu, (unsigned)top);
    const int r_w = __reduce_max_sync(0xFFFFFFFFu, (unsigned)r);
    const int need = bases_needed(n);  // >= 6: bases 2 (done) and 3 always run
    const bool prime = __all_sync(0xFFFFFFFFu, n < (1ull << 63))
                           ? sprp_bases_3_on<true>(M, d, r, top_w, r_w, need)
                           : sprp_bases_3_on<false>(M, d, r, top_w, r_w, need);
    if (live) out[i] = prime ? 1 : 0;
  }
}

// Gap proofs: one warp per gap.  Interior integers are split over the lanes; an interior odd
// integer is marked by the reference's sieve iff it has an odd prime factor q <= isqrt(p_after),
// i.e. iff it is composite or itself a prime <= isqrt(p_after).
__device__ __forceinline__ uint64_t isqrt64(uint64_t x) {
  uint64_t s = (uint64_t)sqrt((double)x);
  if (s > 0xFFFFFFFFull) s = 0xFFFFFFFFull;
  while (s * s > x) --s;
  while (s < 0xFFFFFFFFull && (s + 1) * (s + 1) <= x) ++s;
  return s;
}

// Endpoints of every gap, [2g] = p_after - gap (as the reference: u64 wrap-around), [2g+1] = p_after.
__global__ void gap_ends_kernel(const uint64_t* __restrict__ p_after, const int32_t* __restrict__ gap,
                                uint64_t count, uint64_t* __restrict__ ends) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < count; g += stride) {
    const uint64_t pa = p_after[g];
    ends[2 * g] = pa - (uint64_t)(int64_t)gap[g];
    ends[2 * g + 1] = pa;
  }
}

constexpr int kProveBlock = 256;
constexpr uint32_t kProveChunk = 256;  // interior odd integers examined per round (list capacity)

// Interior proofs, one warp per gap, after the endpoints have been tested (end_ok).  Per round of
// kProveChunk odd interior integers: trial division by the bases 3..37 on all lanes, the
// undecided integers above isqrt(p_after) are appended to a per-warp list in shared memory, and
// the list is tested 32 at a time by a warp-uniform base-2 strong probable-prime test; only
// integers passing it (primes, or base-2 strong pseudoprimes) take the remaining bases.
__global__ void __launch_bounds__(kProveBlock) prove_interior_kernel(const uint64_t* __restrict__ p_after,
                                                                     const int32_t* __restrict__ gap, uint64_t count,
                                                                     const uint8_t* __restrict__ end_ok,
                                                                     uint8_t* __restrict__ ok) {
  __shared__ uint64_t s_list[kProveBlock / 32][kProveChunk];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  uint64_t* list = s_list[wib];
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t g = (uint64_t)blockIdx.x * (blockDim.x >> 5) + wib; g < count; g += warps) {
    const uint64_t pa = p_after[g];
    const int32_t gp = gap[g];
    const uint64_t pb = pa - (uint64_t)(int64_t)gp;
    bool res = end_ok[2 * g] && end_ok[2 * g + 1];
    if (res && gp >= 2) {
      if ((pb & 1ull) == 0) {
        res = false;  // p_before = 2: the even-index marking leaves interior 4 unmarked
      } else {
        const uint64_t sq = isqrt64(pa);
        const uint64_t n_odd = (uint64_t)(gp - 2) / 2;  // odd integers pb+2 .. pa-2
        bool bad = false;
        for (uint64_t k0 = 0; k0 < n_odd && !bad; k0 += kProveChunk) {
          const uint64_t k1 = n_odd - k0 < kProveChunk ? n_odd : k0 + kProveChunk;
          uint32_t n_list = 0;
          bool small_prime = false;
          for (uint64_t kb = k0; kb < k1; kb += 32) {  // warp-uniform trip count
            const uint64_t k = kb + lane;
            int t = 0;
            uint64_t v = 0;
            if (k < k1) {
              v = pb + 2 + 2 * k;
              if (v > sq) t = trial_phase(v);  // 1: a base prime, 0: has a factor <= 37, -1: undecided
            }
            small_prime |= (t == 1);
            const unsigned m = __ballot_sync(0xFFFFFFFFu, t < 0);
            if (t < 0) list[n_list + (uint32_t)__popc(m & ((1u << lane) - 1u))] = v;
            n_list += (uint32_t)__popc(m);
          }
          __syncwarp();
          bad = __any_sync(0xFFFFFFFFu, small_prime);
          for (uint32_t b0 = 0; b0 < n_list && !bad; b0 += 32) {
            const bool live = b0 + lane < n_list;
            const uint64_t v = list[live ? b0 + lane : b0];  // idle lanes shadow the first entry
            const Mont M = mont_setup(v);
            uint64_t d = v - 1;
            const int r = __ffsll((long long)d) - 1;
            d >>= r;
            const int top = 63 - __clzll(d);
            const int top_w = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)top);
            const int r_w = (int)__reduce_max_sync(0xFFFFFFFFu, (unsigned)r);
            const bool small = __all_sync(0xFFFFFFFFu, v < (1ull << 63));
            const bool prp = small ? sprp_uniform<true>(M, 0, d, r, top_w, r_w, true)
                                   : sprp_uniform<false>(M, 0, d, r, top_w, r_w, true);
            const bool pass = live && prp;
            if (__any_sync(0xFFFFFFFFu, pass)) {
              const bool prime = pass && sprp_rest(M, d, r);
              bad = __any_sync(0xFFFFFFFFu, prime);
            }
          }
          __syncwarp();
        }
        res = !bad;
      }
    }
    if (lane == 0) ok[g] = res ? 1 : 0;
  }
}

static int ensure_mr_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
  const uint64_t bit = 1ull << dev;
  if (g_mr_ready.load() & bit) return 0;
  uint64_t inv[12], lim[12];
  for (int i = 0; i < 12; ++i) {
    const uint64_t b = kBases[i];
    uint64_t x = b;
    if (b & 1) {
      for (int k = 0; k < 5; ++k) x *= 2ull - b * x;
    } else {
      x = 0;
    }
    inv[i] = x;
    lim[i] = ~0ull / b;
  }
  if (cudaMemcpyToSymbol(c_base_inv, inv, sizeof(inv)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_base_lim, lim, sizeof(lim)) != cudaSuccess) return -1;
  g_mr_ready.fetch_or(bit);
  return 0;
}

int launch_mr(const uint64_t* d_n, uint64_t count, uint8_t* d_out, uint32_t* d_work,
              uint32_t* d_nwork, void* stream, int sm_count) {
  if (ensure_mr_tables()) return -1;
  if (count == 0) return 0;
  if (count > 0xFFFFFFFFull) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(d_nwork, 0, 2 * sizeof(uint32_t), s) != cudaSuccess) return -1;
  const int blk = 256;
  uint64_t want = (count + blk - 1) / blk;
  int grid = (int)(want < (uint64_t)sm_count * 16 ? want : (uint64_t)sm_count * 16);
  mr_sieve_kernel<<<grid, kSieveBlock, 0, s>>>(d_n, count, d_out, d_work, d_nwork);
  mr_finish_kernel<<<sm_count * 8, blk, 0, s>>>(d_n, d_out, d_work, d_nwork, (uint32_t)count);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_prove_gaps(const uint64_t* d_p_after, const int32_t* d_gap, uint64_t count, uint8_t* d_ok,
                      uint64_t* d_ends, uint8_t* d_ends_ok, uint32_t* d_work, uint32_t* d_nwork, void* stream,
                      int sm_count) {
  if (ensure_mr_tables()) return -1;
  if (count == 0) return 0;
  if (count > 0x7FFFFFFFull) return -1;
  cudaStream_t s = (cudaStream_t)stream;
  // 1. both endpoints of every gap through the batched Miller-Rabin kernels
  const uint64_t eg = (count + 255) / 256;
  gap_ends_kernel<<<(int)(eg < (uint64_t)sm_count * 8 ? eg : (uint64_t)sm_count * 8), 256, 0, s>>>(d_p_after, d_gap,
                                                                                                   count, d_ends);
  if (launch_mr(d_ends, 2 * count, d_ends_ok, d_work, d_nwork, stream, sm_count)) return -1;
  // 2. interiors
  const uint64_t want = (count + (kProveBlock / 32) - 1) / (kProveBlock / 32);
  const int grid = (int)(want < (uint64_t)sm_count * 8 ? want : (uint64_t)sm_count * 8);
  prove_interior_kernel<<<grid, kProveBlock, 0, s>>>(d_p_after, d_gap, count, d_ends_ok, d_ok);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Peak rate of the Montgomery product on this device: independent squaring chains, every lane
// active, no branches and no memory traffic.  The roofline denominator of the Miller-Rabin
// kernels, which spend their time in the same products (one figure per variant: moduli below
// and above 2^63).
constexpr int kMulmodChains = 8;
constexpr int kMulmodIters = 2048;
constexpr int kMulmodBlock = 256;

template <bool kSmallN>
__global__ void __launch_bounds__(kMulmodBlock) mulmod_probe_kernel(uint64_t nbase, uint64_t* sink) {
  const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t n = nbase | (tid << 1) | 1ull;  // an odd modulus per thread
  const Mont M = mont_setup(n);
  uint64_t x[kMulmodChains];
#pragma unroll
  for (int c = 0; c < kMulmodChains; ++c) x[c] = (M.one >> 1) + (uint64_t)c + 1ull;  // < n
#pragma unroll 1
  for (int i = 0; i < kMulmodIters; ++i) {
#pragma unroll
    for (int c = 0; c < kMulmodChains; ++c) x[c] = kSmallN ? mont_mul_small(x[c], x[c], M) : mont_mul(x[c], x[c], M);
  }
  uint64_t acc = 0;
#pragma unroll
  for (int c = 0; c < kMulmodChains; ++c) acc ^= x[c];
  if (acc == 1ull) sink[0] = acc;  // keeps the chains live; practically never taken
}

template <bool kSmallN>
static int probe_mulmod_one(int sm_count, cudaStream_t s, uint64_t* sink, double* per_s) {
  int occ = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mulmod_probe_kernel<kSmallN>, kMulmodBlock, 0) !=
          cudaSuccess ||
      occ < 1)
    return -1;
  const int grid = sm_count * occ;  // one full wave
  const uint64_t nbase = kSmallN ? (1ull << 62) : (3ull << 62);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1;
  }
  mulmod_probe_kernel<kSmallN><<<grid, kMulmodBlock, 0, s>>>(nbase, sink);  // warm-up
  const int reps = 3;
  cudaEventRecord(e0, s);
  for (int r = 0; r < reps; ++r) mulmod_probe_kernel<kSmallN><<<grid, kMulmodBlock, 0, s>>>(nbase, sink);
  cudaEventRecord(e1, s);
  const cudaError_t st = cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != cudaSuccess || ms <= 0) return -1;
  *per_s = (double)grid * kMulmodBlock * kMulmodChains * kMulmodIters * reps / (ms * 1e-3);
  return 0;
}

int probe_mulmod(int sm_count, void* stream, double* full_per_s, double* small_per_s) {
  cudaStream_t s = (cudaStream_t)stream;
  uint64_t* sink = nullptr;
  if (cudaMalloc(&sink, sizeof(uint64_t)) != cudaSuccess) return -1;
  int rc = probe_mulmod_one<false>(sm_count, s, sink, full_per_s);
  if (rc == 0) rc = probe_mulmod_one<true>(sm_count, s, sink, small_per_s);
  cudaFree(sink);
  return rc;
}

}  // namespace voss

// =====================================================================================
// Miller-Rabin without any allocation (voss_mr_verify_noalloc).
//
// Some callers cannot allocate device memory at call time: a process whose device memory is
// already reserved by another allocator (a framework's caching allocator or a memory pool),
// where cudaMalloc would fail or fragment that pool, and request paths of long-running
// services, where cudaMalloc/cudaFree would synchronize the device and stall other streams.
// The regular entry points allocate (the context at creation, per-call buffers on growth);
// this one needs no context and allocates nothing: its scratch (the survivor work list and
// its counter) is the fixed array below, which every device that loads libvoss.so holds
// until the process exits.
// =====================================================================================
namespace voss {

constexpr uint64_t kNoAllocMaxCount = 1ull << 22;  // candidates per call (16 MiB of scratch)
constexpr uint32_t kNoAllocListOffset = 64;         // counters at [0], [1]; list starts 256 B in

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocMaxCount + kNoAllocListOffset];

static std::mutex g_noalloc_mu;
static uint32_t* g_noalloc_ptr[64];  // device address of g_noalloc_scratch, per device ordinal
static int g_noalloc_sms[64];

}  // namespace voss

namespace voss_detail {
int set_error(int code, const char* msg);
}

extern "C" VOSS_API int voss_mr_verify_noalloc(const uint64_t* d_n, uint64_t count, uint8_t* d_is_prime,
                                               void* stream) {
  using namespace voss;
  char msg[160];
  if (count == 0) return VOSS_OK;
  if (!d_n || !d_is_prime) return voss_detail::set_error(VOSS_ERR_ARG, "NULL device pointer");
  if (count > kNoAllocMaxCount) {
    snprintf(msg, sizeof(msg), "count %llu exceeds the no-allocation limit of %llu candidates per call",
             (unsigned long long)count, (unsigned long long)kNoAllocMaxCount);
    return voss_detail::set_error(VOSS_ERR_ARG, msg);
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return voss_detail::set_error(VOSS_ERR_NODEV, "no current CUDA device");
  uint32_t* scratch = nullptr;
  int sms = 0;
  {
    // set-up, once per device, on the calling thread's current device: the host-side name of
    // the array is not a device address, so the kernel gets the address the runtime reports
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        snprintf(msg, sizeof(msg), "cudaGetSymbolAddress(no-allocation scratch) failed: %s", cudaGetErrorString(e));
        return voss_detail::set_error(VOSS_ERR_CUDA, msg);
      }
      int n = 0;
      if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        return voss_detail::set_error(VOSS_ERR_CUDA, "cannot read the SM count");
      g_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
      g_noalloc_sms[dev] = n;
    }
    scratch = g_noalloc_ptr[dev];
    sms = g_noalloc_sms[dev];
  }
  // launch_mr clears the two list counters (cudaMemsetAsync on `scratch`) before its kernels;
  // the list needs no clearing since entries are written before they are read.
  if (launch_mr(d_n, count, d_is_prime, scratch + kNoAllocListOffset, scratch, stream, sms) != 0) {
    snprintf(msg, sizeof(msg), "Miller-Rabin launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    return voss_detail::set_error(VOSS_ERR_CUDA, msg);
  }
  return VOSS_OK;
}

// short_iv.cu — short intervals at high starts by Miller-Rabin instead of the sieve.
//
// Sieving [lo, hi) reduces lo modulo every base prime up to isqrt(hi - 1): at hi = 10^16 that
// is 5.76e6 reductions however short the interval, and at 10^18 50.8e6.  Testing the
// interval's wheel integers (coprime to 30) with the deterministic Miller-Rabin kernels costs
// about 30 Montgomery products per integer instead, so voss_sieve_intervals sends an interval
// here when its base primes above the large-prime threshold outnumber mr_route times its
// length.  The verdicts are exact for every n < 2^64 (mr_kernels.cu), so the statistics are the
// ones the sieve gives: primes >= 7 of [lo, hi), their gap histogram (bin g/2), first and last
// prime, and the first maximal gap.
#include <cuda_runtime.h>

#include <cstdint>

#include "voss.h"
#include "voss_internal.h"

namespace voss {

namespace {

constexpr int kShortBlock = 256;

__device__ __forceinline__ uint64_t wheel_value(const ShortInterval& I, uint32_t j) {
  const uint32_t J = I.j0 + j;
  return I.base + 30ull * (J >> 3) + ((kW30Packed >> (8u * (J & 7u))) & 0xFFu);
}

// The wheel integers of every short interval, in order, at cand[cand_off ...].
__global__ void short_cand_kernel(const ShortInterval* __restrict__ iv, uint32_t n_iv, uint64_t* __restrict__ cand) {
  for (uint32_t b = blockIdx.x; b < n_iv; b += gridDim.x) {
    const ShortInterval I = iv[b];
    for (uint32_t j = threadIdx.x; j < I.n_cand; j += blockDim.x) cand[I.cand_off + j] = wheel_value(I, j);
  }
}

__device__ __forceinline__ void add_gap(uint32_t* hist, uint32_t* over, uint64_t g) {
  if (g < 2ull * VOSS_IHIST)
    atomicAdd(hist + (g >> 1), 1u);
  else
    atomicAdd(over, 1u);
}

// A block per interval: its candidates are split into one contiguous chunk per thread, walked
// in order; the gap into each chunk comes from the last prime of the nearest earlier chunk
// (an exclusive max-scan: primes increase with the chunk index).  Ties of the maximal gap go
// to the smaller lower prime, as in the sieve path.
__global__ void __launch_bounds__(kShortBlock) short_stats_kernel(const ShortInterval* __restrict__ iv,
                                                                  uint32_t n_iv, const uint8_t* __restrict__ ok,
                                                                  voss_interval_stats* __restrict__ out) {
  __shared__ uint32_t hist[VOSS_IHIST];
  __shared__ uint32_t over;
  __shared__ unsigned long long w_scan[kShortBlock / 32];
  __shared__ unsigned long long w_first[kShortBlock / 32];
  __shared__ unsigned long long w_last[kShortBlock / 32];
  __shared__ unsigned long long w_glo[kShortBlock / 32];
  __shared__ uint32_t w_g[kShortBlock / 32];
  __shared__ uint32_t w_cnt[kShortBlock / 32];
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
  constexpr unsigned kFull = 0xFFFFFFFFu;
  for (uint32_t b = blockIdx.x; b < n_iv; b += gridDim.x) {
    const ShortInterval I = iv[b];
    for (uint32_t i = tid; i < (uint32_t)VOSS_IHIST; i += kShortBlock) hist[i] = 0;
    if (tid == 0) over = 0;
    __syncthreads();
    const uint64_t n = I.n_cand;
    const uint64_t per = (n + kShortBlock - 1) / kShortBlock;
    const uint64_t c0 = (uint64_t)tid * per < n ? (uint64_t)tid * per : n;
    const uint64_t c1 = c0 + per < n ? c0 + per : n;
    uint32_t cnt = 0, mg = 0;
    uint64_t first = 0, last = 0, mlo = 0;
    for (uint64_t j = c0; j < c1; ++j) {
      if (!ok[I.cand_off + j]) continue;
      const uint64_t v = wheel_value(I, (uint32_t)j);
      if (cnt) {
        const uint64_t g = v - last;
        add_gap(hist, &over, g);
        if (g > mg) {
          mg = (uint32_t)g;
          mlo = last;
        }
      } else {
        first = v;
      }
      last = v;
      ++cnt;
    }
    // last prime of the nearest earlier chunk that has one (0: none)
    unsigned long long incl = last;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long t = __shfl_up_sync(kFull, incl, d);
      if (lane >= (uint32_t)d && t > incl) incl = t;
    }
    if (lane == 31) w_scan[warp] = incl;
    __syncthreads();
    unsigned long long ex = __shfl_up_sync(kFull, incl, 1);
    if (lane == 0) ex = 0;
    for (uint32_t w = 0; w < warp; ++w) ex = w_scan[w] > ex ? w_scan[w] : ex;
    if (cnt && ex) {
      const uint64_t g = first - ex;
      add_gap(hist, &over, g);
      if (g >= mg) {  // this gap precedes every gap inside the chunk
        mg = (uint32_t)g;
        mlo = ex;
      }
    }
    // block totals: count, first prime (smallest non-zero first), last prime (largest last),
    // maximal gap with the smallest lower prime
    uint32_t tc = cnt;
    unsigned long long tf = cnt ? first : ~0ull, tl = last, glo = mg ? mlo : ~0ull;
    uint32_t tg = mg;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      tc += __shfl_down_sync(kFull, tc, d);
      const unsigned long long f2 = __shfl_down_sync(kFull, tf, d);
      const unsigned long long l2 = __shfl_down_sync(kFull, tl, d);
      const uint32_t g2 = __shfl_down_sync(kFull, tg, d);
      const unsigned long long lo2 = __shfl_down_sync(kFull, glo, d);
      tf = f2 < tf ? f2 : tf;
      tl = l2 > tl ? l2 : tl;
      if (g2 > tg || (g2 == tg && lo2 < glo)) {
        tg = g2;
        glo = lo2;
      }
    }
    if (lane == 0) {
      w_cnt[warp] = tc;
      w_first[warp] = tf;
      w_last[warp] = tl;
      w_g[warp] = tg;
      w_glo[warp] = glo;
    }
    __syncthreads();
    voss_interval_stats* s = out + I.out_index;
    if (tid == 0) {
      uint32_t c = 0, g = 0;
      unsigned long long f = ~0ull, l = 0, lo = ~0ull;
      for (uint32_t w = 0; w < kShortBlock / 32; ++w) {
        c += w_cnt[w];
        f = w_first[w] < f ? w_first[w] : f;
        l = w_last[w] > l ? w_last[w] : l;
        if (w_g[w] > g || (w_g[w] == g && w_glo[w] < lo)) {
          g = w_g[w];
          lo = w_glo[w];
        }
      }
      s->lo = 0;
      s->hi = 0;
      s->prime_count = c;
      s->first_prime = c ? f : 0;
      s->last_prime = c ? l : 0;
      s->max_gap = g;
      s->max_gap_lo = g ? lo : 0;
      s->gap_overflow = over;
    }
    for (uint32_t i = tid; i < (uint32_t)VOSS_IHIST; i += kShortBlock) s->gap_hist[i] = hist[i];
    __syncthreads();  // hist, over and the warp scratch are reused by the next interval
  }
}

}  // namespace

int launch_short_intervals(const ShortInterval* d_iv, uint32_t n_iv, uint64_t n_cand, uint64_t* d_cand,
                           uint8_t* d_ok, uint32_t* d_work, uint32_t* d_nwork, voss_interval_stats* d_out,
                           int sm_count, void* stream) {
  if (n_iv == 0) return 0;
  cudaStream_t s = (cudaStream_t)stream;
  const uint32_t grid = n_iv < (uint32_t)sm_count * 8u ? n_iv : (uint32_t)sm_count * 8u;
  if (n_cand) {
    short_cand_kernel<<<grid, kShortBlock, 0, s>>>(d_iv, n_iv, d_cand);
    if (launch_mr(d_cand, n_cand, d_ok, d_work, d_nwork, stream, sm_count)) return -1;
  }
  short_stats_kernel<<<grid, kShortBlock, 0, s>>>(d_iv, n_iv, d_ok, d_out);
  return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace voss

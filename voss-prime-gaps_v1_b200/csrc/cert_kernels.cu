// cert_kernels.cu — batched SHA-256 on sm_100a for the gap certificates.
//
// The reference's certificate generator (scripts/generate_certificates.py:105-108) hashes one
// short string per large gap, "VOSS|p_before|p_after|gap|merit", with hashlib.sha256, one at a
// time in Python.  Here all messages of a batch are hashed by one kernel, a thread per message,
// following the SHA-256 definition of FIPS 180-4: padding to a multiple of 64 bytes with 0x80,
// zeros and the 64-bit big-endian bit length; the 64-round compression with the message
// schedule kept in a 16-word ring; initial hash value and round constants taken as the first 32
// bits of the fractional parts of the square roots of the first 8 primes and of the cube roots of
// the first 64 primes, which the host computes exactly in integer arithmetic at set-up.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>

#include "voss.h"
#include "voss_host.h"

namespace voss {

__constant__ uint32_t c_sha_k[64];
__constant__ uint32_t c_sha_h0[8];

static std::atomic<uint64_t> g_sha_ready{0};  // per device ordinal

// floor(x^(1/k)) for k = 2, 3 and x < 2^120, by bisection on 128-bit integers.
static uint64_t iroot(unsigned __int128 x, int k) {
  uint64_t lo = 0, hi = 1ull << 41;
  while (hi - lo > 1) {
    const uint64_t mid = lo + (hi - lo) / 2;
    unsigned __int128 p = mid;
    for (int i = 1; i < k; ++i) p *= mid;
    if (p <= x) lo = mid; else hi = mid;
  }
  return lo;
}

static int ensure_sha_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
  const uint64_t bit = 1ull << dev;
  if (g_sha_ready.load() & bit) return 0;
  uint32_t primes[64];
  for (int n = 2, c = 0; c < 64; ++n) {
    bool pr = true;
    for (int d = 2; d * d <= n; ++d)
      if (n % d == 0) pr = false;
    if (pr) primes[c++] = (uint32_t)n;
  }
  uint32_t k[64], h0[8];
  // fractional bits: floor(p^(1/3) * 2^32) = floor((p * 2^96)^(1/3)); keep the low 32 bits
  for (int i = 0; i < 64; ++i) k[i] = (uint32_t)iroot((unsigned __int128)primes[i] << 96, 3);
  for (int i = 0; i < 8; ++i) h0[i] = (uint32_t)iroot((unsigned __int128)primes[i] << 64, 2);
  if (cudaMemcpyToSymbol(c_sha_k, k, sizeof(k)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(c_sha_h0, h0, sizeof(h0)) != cudaSuccess) return -1;
  g_sha_ready.fetch_or(bit);
  return 0;
}

__device__ __forceinline__ uint32_t rotr(uint32_t x, uint32_t n) { return __funnelshift_r(x, x, n); }

// Message i is data[off[i] .. off[i+1]); its digest goes to out[32 i .. 32 i + 32).
__global__ void sha256_batch_kernel(const uint8_t* __restrict__ data, const uint64_t* __restrict__ off,
                                    uint64_t count, uint8_t* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
    const uint64_t base = off[i], len = off[i + 1] - base;
    const uint8_t* m = data + base;
    uint32_t h[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) h[j] = c_sha_h0[j];
    const uint64_t nblk = (len + 9 + 63) / 64;
    const uint64_t bits = len * 8;
    for (uint64_t blk = 0; blk < nblk; ++blk) {
      const bool last = blk + 1 == nblk;
      uint32_t w[16];
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        uint32_t v = 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const uint32_t pos = 4u * t + j;
          const uint64_t idx = blk * 64 + pos;
          uint32_t byte;
          if (idx < len) byte = m[idx];
          else if (idx == len) byte = 0x80u;
          else if (last && pos >= 56) byte = (uint32_t)((bits >> (8 * (63 - pos))) & 0xFFu);
          else byte = 0;
          v = (v << 8) | byte;
        }
        w[t] = v;
      }
      uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
#pragma unroll
      for (int t = 0; t < 64; ++t) {
        if (t >= 16) {
          const uint32_t x15 = w[(t - 15) & 15], x2 = w[(t - 2) & 15];
          const uint32_t s0 = rotr(x15, 7) ^ rotr(x15, 18) ^ (x15 >> 3);
          const uint32_t s1 = rotr(x2, 17) ^ rotr(x2, 19) ^ (x2 >> 10);
          w[t & 15] += s0 + w[(t - 7) & 15] + s1;
        }
        const uint32_t S1 = rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25);
        const uint32_t ch = (e & f) ^ (~e & g);
        const uint32_t t1 = hh + S1 + ch + c_sha_k[t] + w[t & 15];
        const uint32_t S0 = rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22);
        const uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        const uint32_t t2 = S0 + mj;
        hh = g;
        g = f;
        f = e;
        e = d + t1;
        d = c;
        c = b;
        b = a;
        a = t1 + t2;
      }
      h[0] += a;
      h[1] += b;
      h[2] += c;
      h[3] += d;
      h[4] += e;
      h[5] += f;
      h[6] += g;
      h[7] += hh;
    }
    uint8_t* o = out + 32 * i;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      o[4 * j] = (uint8_t)(h[j] >> 24);
      o[4 * j + 1] = (uint8_t)(h[j] >> 16);
      o[4 * j + 2] = (uint8_t)(h[j] >> 8);
      o[4 * j + 3] = (uint8_t)h[j];
    }
  }
}

}  // namespace voss

using namespace voss_host;

extern "C" {

VOSS_API int voss_sha256_batch(voss_ctx* c, const uint8_t* data, const uint64_t* offsets, uint64_t count,
                               uint8_t* digests) {
  NvtxRange nvtx_("voss_sha256_batch");
  if (!c) return fail(VOSS_ERR_ARG, "ctx is NULL");
  if (count == 0) return VOSS_OK;
  if (!offsets || !digests) return fail(VOSS_ERR_ARG, "NULL argument");
  if (offsets[0] != 0) return fail(VOSS_ERR_ARG, "offsets[0] must be 0");
  for (uint64_t i = 0; i < count; ++i)
    if (offsets[i + 1] < offsets[i]) return fail(VOSS_ERR_ARG, "offsets must not decrease (entry %llu)",
                                                 (unsigned long long)i);
  const uint64_t bytes = offsets[count];
  if (bytes && !data) return fail(VOSS_ERR_ARG, "NULL data");
  cudaSetDevice(c->device);
  if (voss::ensure_sha_tables()) return fail(VOSS_ERR_CUDA, "SHA-256 constant upload failed");
  cudaStream_t s = c->stream;
  Workspace& W = c->ws;  // context-owned, grow-only buffers
  int rc;
  if ((rc = W.sha_data.ensure(std::max<uint64_t>(bytes, 1))) || (rc = W.sha_off.ensure(8 * (count + 1))) ||
      (rc = W.sha_out.ensure(32 * count)))
    return rc;
  if (bytes) CUDA_TRY(cudaMemcpyAsync(W.sha_data.p, data, bytes, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(W.sha_off.p, offsets, 8 * (count + 1), cudaMemcpyHostToDevice, s));
  const uint64_t want = (count + 127) / 128;
  const int grid = (int)std::min<uint64_t>(want, (uint64_t)c->sm_count * 16);
  voss::sha256_batch_kernel<<<grid, 128, 0, s>>>(W.sha_data.as<uint8_t>(), W.sha_off.as<uint64_t>(), count,
                                                 W.sha_out.as<uint8_t>());
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(digests, W.sha_out.p, 32 * count, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return VOSS_OK;
}

}  // extern "C"

// ref_verify_shim.cpp — exposes the reference verifier's functions through a C ABI.
//
// TEST INFRASTRUCTURE ONLY: built by oracle/Makefile into oracle/_ref/libref_verify.so from
// the reference's own, unmodified src/verify_cpp.cpp (included below from the reference tree,
// never copied), and loaded only by tests/ and bench.py's reference arm as the checker and
// the timed CPU baseline.  Its static functions is_prime_u64 (verify_cpp.cpp:38-57),
// verify_gap (:59-93) and build_base_sieve (:95-103) become callable; its main() is renamed
// so that it is not the program entry point.
#define main verify_cpp_main
#include "verify_cpp.cpp"
#undef main

#include <omp.h>

extern "C" {

int ref_is_prime_u64(uint64_t n) { return is_prime_u64(n) ? 1 : 0; }

void ref_mr_batch(const uint64_t* n, uint64_t count, uint8_t* out, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t i = 0; i < (int64_t)count; i++) out[i] = is_prime_u64(n[i]) ? 1 : 0;
}

// verify_cpp's main loop body (verify_cpp.cpp:180-217) without its CSV I/O, cache and the
// 30-second monitor thread: one base sieve up to isqrt(max p_after) + 1, then verify_gap
// for every gap under OpenMP with the same schedule(dynamic, 64).
void ref_prove_gaps(const uint64_t* p_after, const int32_t* gap, uint64_t count, uint8_t* ok,
                    int threads) {
  u64 max_p = 0;
  for (uint64_t i = 0; i < count; i++) if (p_after[i] > max_p) max_p = p_after[i];
  u64 limit = (u64)sqrtl((long double)max_p) + 1;
  std::vector<uint32_t> bp = build_base_sieve(limit);
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < (int64_t)count; i++) ok[i] = verify_gap(p_after[i], gap[i], bp) ? 1 : 0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"

/*
 * sieve_oracle.c — CPU oracle for the VOSS sieve-and-gap path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load this code (as liboracle.so), and only as the checker or the timed CPU
 * baseline; the product library (libvoss.so) never links or calls it.
 *
 * It restates, in plain C + OpenMP, the reference's CPU algorithms:
 *   - build_base_sieve             src/verify_cpp.cpp:95-103
 *   - mul_mod / mod_pow / is_prime_u64 (12 bases)   src/verify_cpp.cpp:24-57
 *   - verify_gap (interval-composite proof)         src/verify_cpp.cpp:59-93
 *   - an interval sieve that applies verify_gap's marking loop (evens, then odd multiples
 *     of each odd base prime q with stride 2q, verify_cpp.cpp:73-90) to consecutive
 *     windows, starting each prime at max(q*q, window start) so that q itself survives,
 * and feeds the primes, in order, through the statistics rules of src/voss_v7_live.cu:
 *   gap histogram (:278-280, :559-561, :634-635), mod-4 (:181-193, :682),
 *   mod-q (:195-232), per-residue gap histogram (:282-287), large gaps (:289-299),
 *   segment-boundary exclusion of the reference-compat mode (:551-562).
 * Parity of this restatement is pinned by tests/test_oracle.py against the reference's
 * committed golden vectors (results/hist_snapshots, data/verification_db.json,
 * README Chebyshev table) and against the reference verify_cpp.cpp compiled unmodified
 * (oracle/_ref/libref_verify.so).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "voss.h"

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* Miller-Rabin: restates src/verify_cpp.cpp:24-57                             */
/* ------------------------------------------------------------------------- */
static inline uint64_t o_mul_mod(uint64_t a, uint64_t b, uint64_t m) {
  return (uint64_t)((u128)a * b % m);
}

static inline uint64_t o_mod_pow(uint64_t base, uint64_t exp, uint64_t mod) {
  uint64_t result = 1;
  base %= mod;
  while (exp > 0) {
    if (exp & 1) result = o_mul_mod(result, base, mod);
    base = o_mul_mod(base, base, mod);
    exp >>= 1;
  }
  return result;
}

static const uint64_t O_BASES[12] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};

int oracle_is_prime_u64(uint64_t n) {
  if (n < 2) return 0;
  for (int i = 0; i < 12; i++) {
    if (n == O_BASES[i]) return 1;
    if (n % O_BASES[i] == 0) return 0;
  }
  uint64_t d = n - 1;
  int r = 0;
  while ((d & 1) == 0) { d >>= 1; r++; }
  for (int i = 0; i < 12; i++) {
    uint64_t x = o_mod_pow(O_BASES[i], d, n);
    if (x == 1 || x == n - 1) continue;
    int composite = 1;
    for (int j = 0; j < r - 1; j++) {
      x = o_mul_mod(x, x, n);
      if (x == n - 1) { composite = 0; break; }
    }
    if (composite) return 0;
  }
  return 1;
}

void oracle_mr_batch(const uint64_t* n, uint64_t count, uint8_t* out, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4096)
#endif
  for (int64_t i = 0; i < (int64_t)count; i++) out[i] = (uint8_t)oracle_is_prime_u64(n[i]);
}

/* ------------------------------------------------------------------------- */
/* Base primes: restates build_base_sieve, src/verify_cpp.cpp:95-103           */
/* ------------------------------------------------------------------------- */
static uint64_t o_isqrt(uint64_t x) {
  /* the reference's exact integer square root (verify_cpp.cpp:75-77) */
  uint64_t s = (uint64_t)sqrtl((long double)x);
  while ((s + 1) * (s + 1) <= x) s++;
  while (s * s > x) s--;
  return s;
}

/* All primes <= limit, ascending (the list build_base_sieve makes, verify_cpp.cpp:95-103).
 * Small limits use the plain sieve of a byte per integer; above 2^24 the odd integers are
 * sieved in segments of 2^21 by the primes up to sqrt(limit), so that limits near 2^31
 * (intervals just below 2^62) take seconds rather than a minute of cache misses. */
uint32_t* oracle_base_primes(uint64_t limit, uint64_t* count) {
  if (limit <= (1u << 24)) {
    uint8_t* s = (uint8_t*)malloc(limit + 1);
    if (!s) { *count = 0; return NULL; }
    memset(s, 1, limit + 1);
    s[0] = 0;
    if (limit >= 1) s[1] = 0;
    for (uint64_t i = 2; i * i <= limit; i++)
      if (s[i])
        for (uint64_t j = i * i; j <= limit; j += i) s[j] = 0;
    uint64_t c = 0;
    for (uint64_t i = 2; i <= limit; i++) c += s[i];
    uint32_t* p = (uint32_t*)malloc((c ? c : 1) * sizeof(uint32_t));
    uint64_t k = 0;
    for (uint64_t i = 2; i <= limit; i++)
      if (s[i]) p[k++] = (uint32_t)i;
    free(s);
    *count = c;
    return p;
  }
  uint64_t nsm = 0;
  uint32_t* sm = oracle_base_primes(o_isqrt(limit), &nsm);
  /* pi(x) < 1.26 x / ln x for x > 1 (Rosser-Schoenfeld): capacity for the whole list */
  uint64_t cap = (uint64_t)(1.26 * (double)limit / log((double)limit)) + 64;
  uint32_t* p = (uint32_t*)malloc(cap * sizeof(uint32_t));
  const uint64_t SEG = 1u << 21; /* odd integers per segment */
  uint8_t* seg = (uint8_t*)malloc(SEG);
  if (!p || !seg || !sm) { free(p); free(seg); free(sm); *count = 0; return NULL; }
  uint64_t k = 0;
  p[k++] = 2;
  for (uint64_t base = 1; base <= limit; base += 2 * SEG) { /* slot i <-> base + 2i */
    uint64_t n = SEG;
    if (base + 2 * (n - 1) > limit) n = (limit - base) / 2 + 1;
    memset(seg, 1, n);
    const uint64_t vmax = base + 2 * (n - 1);
    for (uint64_t t = 1; t < nsm; t++) { /* odd primes */
      const uint64_t q = sm[t];
      if (q * q > vmax) break;
      uint64_t m = q * q;
      if (m < base) {
        m = (base + q - 1) / q * q;
        if ((m & 1) == 0) m += q;
      }
      for (uint64_t i = (m - base) / 2; i < n; i += q) seg[i] = 0;
    }
    for (uint64_t i = 0; i < n; i++)
      if (seg[i] && base + 2 * i > 1) p[k++] = (uint32_t)(base + 2 * i);
  }
  free(seg);
  free(sm);
  *count = k;
  return p;
}

void oracle_free(void* p) { free(p); }

/* ------------------------------------------------------------------------- */
/* verify_gap: restates src/verify_cpp.cpp:59-93 literally                     */
/* ------------------------------------------------------------------------- */
int oracle_verify_gap(uint64_t p_after, int gap, const uint32_t* bp, uint64_t nbp) {
  uint64_t p_before = p_after - (uint64_t)(int64_t)gap;
  if (!oracle_is_prime_u64(p_before)) return 0;
  if (!oracle_is_prime_u64(p_after)) return 0;
  if (gap < 2) return 1;
  int n_int = gap - 1;
  uint8_t stack_buf[1024];
  uint8_t* is_comp = n_int <= 1024 ? stack_buf : (uint8_t*)malloc((size_t)n_int);
  memset(is_comp, 0, (size_t)n_int);
  for (int i = 0; i < n_int; i += 2) is_comp[i] = 1;
  uint64_t sq = o_isqrt(p_after);
  for (uint64_t k = 0; k < nbp; k++) {
    uint64_t q = bp[k];
    if (q == 2) continue;
    if (q > sq) break;
    uint64_t start = (p_before / q + 1) * q;
    if ((start & 1) == 0) start += q;
    if (start >= p_after) continue;
    int64_t idx = (int64_t)(start - p_before - 1);
    if (idx < 0) idx = 0;
    int step = (int)(2 * q);
    for (int i = (int)idx; i < n_int; i += step) is_comp[i] = 1;
  }
  int ok = 1;
  for (int i = 0; i < n_int; i++)
    if (!is_comp[i]) { ok = 0; break; }
  if (is_comp != stack_buf) free(is_comp);
  return ok;
}

void oracle_prove_gaps(const uint64_t* p_after, const int32_t* gap, uint64_t count, uint8_t* ok,
                       int threads) {
  uint64_t maxp = 0;
  for (uint64_t i = 0; i < count; i++)
    if (p_after[i] > maxp) maxp = p_after[i];
  /* verify_cpp.cpp:180-184: one base sieve up to isqrt(max p) + 1 */
  uint64_t nbp = 0;
  uint32_t* bp = oracle_base_primes((uint64_t)sqrtl((long double)maxp) + 1, &nbp);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
  for (int64_t i = 0; i < (int64_t)count; i++)
    ok[i] = (uint8_t)oracle_verify_gap(p_after[i], gap[i], bp, nbp);
  free(bp);
}

/* ------------------------------------------------------------------------- */
/* Interval sieve over windows + statistics                                    */
/* ------------------------------------------------------------------------- */
static const int O_W30[8] = {1, 7, 11, 13, 17, 19, 23, 29};
static const int O_QS[VOSS_NUM_Q] = VOSS_Q_LIST;

static int o_row6(uint64_t p) { return (p % 6) == 1 ? 0 : 1; } /* W30_TO_Q6_IDX, :30 */
static int o_row30(uint64_t p) {                                /* W30_TO_Q30_IDX, :31 */
  int r = (int)(p % 30);
  for (int i = 0; i < 8; i++)
    if (O_W30[i] == r) return i;
  return -1;
}

typedef struct {
  /* configuration */
  int compat;
  uint64_t seg_num;
  int interval_mode;
  /* state */
  uint64_t prev;
  uint64_t count, first, last;
  uint64_t max_gap, max_gap_lo;
  uint64_t mod4[2];
  uint64_t modq[VOSS_MODQ_SLOTS];
  uint64_t* modq_gap; /* [10][100] */
  uint64_t* gap_hist; /* [VOSS_MAX_GAP] or [VOSS_IHIST] in interval mode */
  uint64_t gap_overflow;
  voss_large_gap* large;
  uint64_t n_large, cap_large;
} o_acc;

static void o_acc_init(o_acc* a, int compat, uint64_t seg_num, int interval_mode) {
  memset(a, 0, sizeof(*a));
  a->compat = compat;
  a->seg_num = seg_num;
  a->interval_mode = interval_mode;
  if (!interval_mode) {
    a->modq_gap = (uint64_t*)calloc(VOSS_MODQ_ROWS * VOSS_MODQ_MAX_GAP, sizeof(uint64_t));
    a->gap_hist = (uint64_t*)calloc(VOSS_MAX_GAP, sizeof(uint64_t));
  } else {
    a->gap_hist = (uint64_t*)calloc(VOSS_IHIST, sizeof(uint64_t));
  }
}

static void o_acc_free(o_acc* a) {
  free(a->modq_gap);
  free(a->gap_hist);
  free(a->large);
}

static void o_push_large(o_acc* a, uint64_t pos, int32_t gap, float merit) {
  if (a->n_large == a->cap_large) {
    a->cap_large = a->cap_large ? 2 * a->cap_large : 1024;
    a->large = (voss_large_gap*)realloc(a->large, a->cap_large * sizeof(voss_large_gap));
  }
  a->large[a->n_large].position = pos;
  a->large[a->n_large].gap = gap;
  a->large[a->n_large].merit = merit;
  a->n_large++;
}

/* The statistics of one consecutive pair (lo_p, hi_p). */
static void o_pair(o_acc* a, uint64_t lo_p, uint64_t hi_p) {
  uint64_t g = hi_p - lo_p;
  if (a->interval_mode) {
    if (g < 2 * VOSS_IHIST) a->gap_hist[g >> 1]++;
    else a->gap_overflow++;
  } else if (g < VOSS_MAX_GAP) {
    a->gap_hist[g]++;
  }
  if (g > a->max_gap) { a->max_gap = g; a->max_gap_lo = lo_p; }
  if (a->interval_mode) return;
  if (lo_p < 7) return; /* 2, 3, 5 never enter the wheel kernels (:404) */
  if (a->compat && (lo_p - 1) / a->seg_num != (hi_p - 1) / a->seg_num) return; /* :559-561 */
  if (g < VOSS_MODQ_MAX_GAP) { /* :283-287 */
    a->modq_gap[o_row6(lo_p) * VOSS_MODQ_MAX_GAP + g]++;
    a->modq_gap[(2 + o_row30(lo_p)) * VOSS_MODQ_MAX_GAP + g]++;
  }
  double merit_d = 0.0; /* :289-299 */
  if (g > 100) merit_d = (double)g / log((double)lo_p);
  if (g >= 500 || merit_d >= 10.0)
    if (g < VOSS_MAX_GAP) o_push_large(a, hi_p, (int32_t)g, (float)merit_d);
}

static inline void o_prime(o_acc* a, uint64_t p) {
  a->count++;
  if (!a->first) a->first = p;
  if (!a->interval_mode) {
    int m4 = (int)(p & 3);
    if (m4 == 1) a->mod4[0]++;
    else if (m4 == 3) a->mod4[1]++;
    if (!a->compat || p >= 7) {
      int off = 0;
      for (int qi = 0; qi < VOSS_NUM_Q; qi++) {
        a->modq[off + (int)(p % (uint64_t)O_QS[qi])]++;
        off += O_QS[qi];
      }
    }
  }
  if (a->prev) o_pair(a, a->prev, p);
  a->prev = p;
  a->last = p;
}

/* Sieve [lo, hi) (window by window) feeding primes into `a` in ascending order.
 * bp: all primes up to at least isqrt(hi - 1), including 2. */
static void o_sieve_span(o_acc* a, uint64_t lo, uint64_t hi, const uint32_t* bp, uint64_t nbp) {
  /* Odd slots per window: every window costs one division per base prime up to its isqrt,
   * so windows grow with that count (2^20 .. 2^24 slots) to keep the divisions a small part
   * of the marking at starts near 10^16 .. 10^18 (5.8e6 .. 5.1e7 base primes). */
  uint64_t WIN = 1u << 20;
  {
    uint64_t r = hi > 1 ? o_isqrt(hi - 1) : 1, used = 0;
    uint64_t lo_k = 0, hi_k = nbp; /* number of base primes <= r (bp is ascending) */
    while (lo_k < hi_k) {
      uint64_t mid = (lo_k + hi_k) / 2;
      if (bp[mid] <= r) lo_k = mid + 1; else hi_k = mid;
    }
    used = lo_k;
    while (WIN < used && WIN < (1u << 24)) WIN <<= 1;
  }
  if (lo < 2) lo = 2;
  if (lo >= hi) return;
  if (lo <= 2 && 2 < hi) o_prime(a, 2);
  uint8_t* is_comp = (uint8_t*)malloc(WIN);
  uint64_t base = lo & ~(uint64_t)1; /* even; slot i <-> value base + 2i + 1 */
  while (base + 1 < hi) {
    uint64_t wend = base + 2 * WIN; /* exclusive value bound */
    if (wend > hi || wend < base) wend = hi;
    uint64_t nslots = (wend - base) / 2; /* values base+1 .. base+2*nslots-1 */
    if (nslots == 0) break;
    memset(is_comp, 0, nslots);
    uint64_t vmax = base + 2 * nslots - 1;
    for (uint64_t k = 0; k < nbp; k++) {
      uint64_t q = bp[k];
      if (q == 2) continue;
      if (q * q > vmax) break;
      uint64_t from = base + 1 > q * q ? base + 1 : q * q;
      uint64_t m = (from + q - 1) / q * q;
      if ((m & 1) == 0) m += q;
      for (uint64_t i = (m - base - 1) / 2; i < nslots; i += q) is_comp[i] = 1;
    }
    for (uint64_t i = 0; i < nslots; i++) {
      if (is_comp[i]) continue;
      uint64_t v = base + 2 * i + 1;
      if (v < lo || v < 3) continue;
      o_prime(a, v);
    }
    base = wend & ~(uint64_t)1;
    if (wend == hi) break;
  }
  free(is_comp);
}

/* Merge thread-local accumulators in range order, adding the pair across each seam. */
static void o_merge(o_acc* dst, o_acc* src) {
  if (src->count == 0) return;
  if (dst->count && dst->prev) o_pair(dst, dst->prev, src->first);
  dst->count += src->count;
  if (!dst->first) dst->first = src->first;
  dst->last = src->last;
  dst->prev = src->prev;
  if (src->max_gap > dst->max_gap) { dst->max_gap = src->max_gap; dst->max_gap_lo = src->max_gap_lo; }
  dst->mod4[0] += src->mod4[0];
  dst->mod4[1] += src->mod4[1];
  for (int i = 0; i < VOSS_MODQ_SLOTS; i++) dst->modq[i] += src->modq[i];
  if (!dst->interval_mode) {
    for (int i = 0; i < VOSS_MODQ_ROWS * VOSS_MODQ_MAX_GAP; i++) dst->modq_gap[i] += src->modq_gap[i];
    for (int i = 0; i < VOSS_MAX_GAP; i++) dst->gap_hist[i] += src->gap_hist[i];
  } else {
    for (int i = 0; i < VOSS_IHIST; i++) dst->gap_hist[i] += src->gap_hist[i];
  }
  dst->gap_overflow += src->gap_overflow;
  for (uint64_t i = 0; i < src->n_large; i++)
    o_push_large(dst, src->large[i].position, src->large[i].gap, src->large[i].merit);
}

/* Whole-range statistics with the semantics of voss_sieve_range (include/voss.h). */
int oracle_sieve_range(uint64_t lo, uint64_t hi, uint32_t flags, uint64_t seg_num, int threads,
                       voss_range_stats* st, voss_large_gap* large, uint64_t large_cap,
                       uint64_t* large_written) {
  int compat = (flags & VOSS_FLAG_REF_COMPAT) != 0;
  if (hi < lo) return VOSS_ERR_ARG;
  if (compat && (seg_num == 0 || seg_num % 30 != 0)) return VOSS_ERR_ARG;
  uint64_t nbp = 0;
  uint32_t* bp = oracle_base_primes(hi > 1 ? o_isqrt(hi - 1) + 1 : 2, &nbp);
  int T = 1;
#ifdef _OPENMP
  T = threads > 0 ? threads : omp_get_max_threads();
#endif
  uint64_t span = hi - lo;
  if ((uint64_t)T > span / (1u << 16) + 1) T = (int)(span / (1u << 16) + 1);
  o_acc* acc = (o_acc*)calloc((size_t)T, sizeof(o_acc));
  for (int t = 0; t < T; t++) o_acc_init(&acc[t], compat, seg_num, 0);
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(static, 1)
#endif
  for (int t = 0; t < T; t++) {
    uint64_t a = lo + (uint64_t)((u128)span * (uint64_t)t / (uint64_t)T);
    uint64_t b = lo + (uint64_t)((u128)span * (uint64_t)(t + 1) / (uint64_t)T);
    o_sieve_span(&acc[t], a, b, bp, nbp);
  }
  for (int t = 1; t < T; t++) o_merge(&acc[0], &acc[t]);
  o_acc* A = &acc[0];

  memset(st, 0, sizeof(*st));
  st->lo = lo;
  st->hi = hi;
  st->flags = flags;
  st->seg_num = compat ? seg_num : 0;
  st->prime_count = A->count;
  st->first_prime = A->first;
  st->last_prime = A->last;
  st->max_gap = A->max_gap;
  st->max_gap_lo = A->max_gap_lo;
  st->mod4[0] = A->mod4[0];
  st->mod4[1] = A->mod4[1];
  memcpy(st->modq, A->modq, sizeof(st->modq));
  memcpy(st->modq_gap, A->modq_gap, sizeof(st->modq_gap));
  memcpy(st->gap_hist, A->gap_hist, sizeof(st->gap_hist));
  st->large_total = A->n_large;
  uint64_t w = A->n_large < large_cap ? A->n_large : large_cap;
  if (large && w) memcpy(large, A->large, w * sizeof(voss_large_gap));
  if (large_written) *large_written = w;
  for (int t = 0; t < T; t++) o_acc_free(&acc[t]);
  free(acc);
  free(bp);
  return VOSS_OK;
}

/* Per-interval statistics with the semantics of voss_sieve_intervals.  Each interval is cut
 * into chunks of at most O_IV_CHUNK integers; the chunks of all intervals run in parallel
 * and are merged per interval in order (o_merge adds the gap across each seam), so one
 * interval of 10^8 integers is not left to a single thread. */
#define O_IV_CHUNK ((uint64_t)1 << 24)
int oracle_sieve_intervals(const uint64_t* lo, const uint64_t* hi, uint32_t n, int threads,
                           voss_interval_stats* out) {
  uint64_t maxhi = 2;
  for (uint32_t i = 0; i < n; i++) {
    if (hi[i] < lo[i]) return VOSS_ERR_ARG;
    if (hi[i] > maxhi) maxhi = hi[i];
  }
  uint64_t nbp = 0;
  uint32_t* bp = oracle_base_primes(o_isqrt(maxhi - 1) + 1, &nbp);
  /* chunk c of interval i covers [lo_i + c*O_IV_CHUNK, min(hi_i, lo_i + (c+1)*O_IV_CHUNK)) */
  uint64_t* first_chunk = (uint64_t*)malloc(((size_t)n + 1) * sizeof(uint64_t));
  uint64_t total = 0;
  for (uint32_t i = 0; i < n; i++) {
    first_chunk[i] = total;
    uint64_t len = hi[i] - lo[i];
    total += len ? (len + O_IV_CHUNK - 1) / O_IV_CHUNK : 1;
  }
  first_chunk[n] = total;
  uint32_t* owner = (uint32_t*)malloc((size_t)(total ? total : 1) * sizeof(uint32_t));
  for (uint32_t i = 0; i < n; i++)
    for (uint64_t c = first_chunk[i]; c < first_chunk[i + 1]; c++) owner[c] = i;
  o_acc* acc = (o_acc*)calloc((size_t)(total ? total : 1), sizeof(o_acc));
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t c = 0; c < (int64_t)total; c++) {
    uint32_t i = owner[c];
    uint64_t a = lo[i] + (uint64_t)(c - (int64_t)first_chunk[i]) * O_IV_CHUNK;
    uint64_t b = hi[i] - a > O_IV_CHUNK ? a + O_IV_CHUNK : hi[i];
    o_acc_init(&acc[c], 0, 0, 1);
    o_sieve_span(&acc[c], a, b, bp, nbp);
  }
  for (uint32_t i = 0; i < n; i++) {
    o_acc* A = &acc[first_chunk[i]];
    for (uint64_t c = first_chunk[i] + 1; c < first_chunk[i + 1]; c++) o_merge(A, &acc[c]);
    voss_interval_stats* s = &out[i];
    memset(s, 0, sizeof(*s));
    s->lo = lo[i];
    s->hi = hi[i];
    s->prime_count = A->count;
    s->first_prime = A->first;
    s->last_prime = A->last;
    s->max_gap = A->max_gap;
    s->max_gap_lo = A->max_gap_lo;
    s->gap_overflow = A->gap_overflow;
    memcpy(s->gap_hist, A->gap_hist, sizeof(s->gap_hist));
  }
  for (uint64_t c = 0; c < total; c++) o_acc_free(&acc[c]);
  free(acc);
  free(owner);
  free(first_chunk);
  free(bp);
  return VOSS_OK;
}

/* Primes of [lo, hi) in ascending order (single thread; test sizes only). */
typedef struct {
  uint64_t* out;
  uint64_t cap, n;
} o_list;

int oracle_primes_range(uint64_t lo, uint64_t hi, uint64_t* out, uint64_t cap, uint64_t* count) {
  uint64_t nbp = 0;
  uint32_t* bp = oracle_base_primes(hi > 1 ? o_isqrt(hi - 1) + 1 : 2, &nbp);
  uint64_t n = 0;
  const uint64_t WIN = 1u << 20;
  uint8_t* is_comp = (uint8_t*)malloc(WIN);
  if (lo < 2) lo = 2;
  if (lo <= 2 && 2 < hi) { if (n < cap) out[n] = 2; n++; }
  uint64_t base = lo & ~(uint64_t)1;
  while (lo < hi && base + 1 < hi) {
    uint64_t wend = base + 2 * WIN;
    if (wend > hi || wend < base) wend = hi;
    uint64_t nslots = (wend - base) / 2;
    if (nslots == 0) break;
    memset(is_comp, 0, nslots);
    uint64_t vmax = base + 2 * nslots - 1;
    for (uint64_t k = 0; k < nbp; k++) {
      uint64_t q = bp[k];
      if (q == 2) continue;
      if (q * q > vmax) break;
      uint64_t from = base + 1 > q * q ? base + 1 : q * q;
      uint64_t m = (from + q - 1) / q * q;
      if ((m & 1) == 0) m += q;
      for (uint64_t i = (m - base - 1) / 2; i < nslots; i += q) is_comp[i] = 1;
    }
    for (uint64_t i = 0; i < nslots; i++) {
      uint64_t v = base + 2 * i + 1;
      if (is_comp[i] || v < lo || v < 3) continue;
      if (n < cap) out[n] = v;
      n++;
    }
    base = wend & ~(uint64_t)1;
    if (wend == hi) break;
  }
  free(is_comp);
  free(bp);
  *count = n;
  return VOSS_OK;
}

/* H(N): number of bit-clears of a wheel-30 sieve of [1, N] that clears, for every prime
 * 7 <= p <= isqrt(N), the multiples p*m with m >= p and gcd(m, 30) = 1 — the algorithmic
 * unit of work of src/voss_v7_live.cu:120-143 (one atomicAnd per (p, multiple)). */
static uint64_t o_coprime30_upto(uint64_t x) { /* #{1 <= m <= x : gcd(m,30)=1} */
  uint64_t c = (x / 30) * 8;
  uint64_t r = x % 30;
  for (int i = 0; i < 8; i++)
    if ((uint64_t)O_W30[i] <= r) c++;
  return c;
}

uint64_t oracle_sieve_work(uint64_t N) {
  uint64_t nbp = 0;
  uint64_t s = o_isqrt(N);
  uint32_t* bp = oracle_base_primes(s + 1, &nbp);
  uint64_t h = 0;
  for (uint64_t k = 0; k < nbp; k++) {
    uint64_t p = bp[k];
    if (p < 7) continue;
    if (p * p > N) break;
    h += o_coprime30_upto(N / p) - o_coprime30_upto(p - 1);
  }
  free(bp);
  return h;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/*
 * voss.h — C ABI of the B200-native VOSS sieve-and-gap engine (libvoss.so).
 *
 * The reference (atafhamada/voss-prime-gaps_v1) has no library interface: its hot
 * path is the stand-alone program src/voss_v7_live.cu, configured by regex-patched
 * compile-time constants (src/voss_master.py:64-85) and reporting through CSV files
 * and stdout, plus the verifier program src/verify_cpp.cpp driven by argv.  Each
 * entry point below replaces one of those interfaces; the comment on each names the
 * reference lines it stands in for.
 *
 * Conventions
 *   - every function returns int: VOSS_OK (0) or a negative VOSS_ERR_* code; the
 *     library never calls exit() (the reference exits via CUDA_CHECK,
 *     src/voss_v7_live.cu:17-21, and on MAX_POS overflow, :516-519);
 *   - voss_last_error() gives a message for the last failure on this thread;
 *   - all pointers in signatures are HOST pointers owned by the caller, except the
 *     *_device entry points, which say so; no pointer is retained after return;
 *   - integer ranges are half-open [lo, hi); the reference's N-inclusive range
 *     [1, N] (src/voss_v7_live.cu:435-445) is lo = 1, hi = N + 1;
 *   - a context is bound to one CUDA device and is used by one host thread at a
 *     time; use one context per thread.
 */
#ifndef VOSS_H
#define VOSS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define VOSS_API __attribute__((visibility("default")))
#else
#define VOSS_API
#endif

/* ---- error codes ---------------------------------------------------------- */
#define VOSS_OK 0
#define VOSS_ERR_ARG (-1)      /* invalid argument */
#define VOSS_ERR_CUDA (-2)     /* a CUDA runtime call failed */
#define VOSS_ERR_NOMEM (-3)    /* device or host allocation failed */
#define VOSS_ERR_RANGE (-4)    /* hi beyond the context's base-prime limit */
#define VOSS_ERR_DEVICE (-5)   /* a kernel raised its error word */
#define VOSS_ERR_TIMEOUT (-6)  /* a bounded wait ran out */
#define VOSS_ERR_STOPPED (-7)  /* stop file seen; checkpoint written */
#define VOSS_ERR_IO (-8)       /* file could not be read or written */
#define VOSS_ERR_STATE (-9)    /* object in the wrong state for the call */
#define VOSS_ERR_NODEV (-10)   /* no CUDA device */

/* ---- sizes shared with the reference's artifact formats ------------------- */
#define VOSS_MAX_GAP 100000    /* gap histogram covers 0 < g < 1e5: voss_v7_live.cu:23,280 */
#define VOSS_MODQ_MAX_GAP 100  /* per-residue gap histogram: g < 100: voss_v7_live.cu:25,283 */
#define VOSS_MODQ_ROWS 10      /* rows: q=6 residues {1,5}, then q=30 residues W30: :26-31,758-764 */
#define VOSS_NUM_Q 10          /* moduli of voss_range_stats.modq, see VOSS_Q_LIST */
#define VOSS_MODQ_SLOTS 99     /* 3+4+5+6+7+8+11+12+13+30 */
#define VOSS_Q_LIST {3, 4, 5, 6, 7, 8, 11, 12, 13, 30}
#define VOSS_IHIST 1024        /* per-interval gap bins: bin g/2 holds gap g (bin 0 holds g = 1) */

/* voss_range_stats.flags */
#define VOSS_FLAG_REF_COMPAT 1u /* reproduce voss_v7_live's artifact rules exactly (see below) */

/* One large gap, layout of `struct LargeGap` (src/voss_v7_live.cu:40): position is the
 * upper prime p_after, merit = (float)(gap / log(p_before)) computed in double. */
typedef struct voss_large_gap {
  uint64_t position;
  int32_t gap;
  float merit;
} voss_large_gap;

/*
 * Whole-range statistics: every array the reference accumulates for its CSVs
 * (src/voss_v7_live.cu:403-405, 581-594, 634-635, 737-771).
 *
 * Full mode (flags = 0): every quantity covers exactly the primes in [lo, hi):
 *   prime_count, gap_hist over consecutive pairs inside the range, mod4 and modq over
 *   all primes in range; modq_gap and the large-gap list over pairs whose lower prime
 *   is >= 7 (the rows of modq_gap are residues coprime to 30).
 * Reference-compat mode (VOSS_FLAG_REF_COMPAT, lo must be 1): the numbers voss_v7_live
 *   prints and writes for N = hi - 1 with segment length seg_num:
 *   - 2, 3, 5 are counted in prime_count, gap_hist (gaps 1, 2 and the 5->7 gap) and
 *     mod4 (3 and 5), but not in modq, modq_gap or the large-gap list (:404,634-635,682);
 *   - a gap between primes in different segments [s*seg_num+1, (s+1)*seg_num] enters
 *     gap_hist only, not modq_gap nor the large-gap list (:559-562).
 */
typedef struct voss_range_stats {
  uint64_t lo, hi;          /* [lo, hi) */
  uint32_t flags;           /* VOSS_FLAG_* used */
  uint32_t reserved0;
  uint64_t seg_num;         /* compat segment length (integers), 0 in full mode */
  uint64_t prime_count;     /* pi(hi-1) - pi(lo-1); "Total primes" (:639) */
  uint64_t first_prime;     /* 0 if no prime in range */
  uint64_t last_prime;      /* 0 if no prime in range; "p_last" (:700) */
  uint64_t max_gap;         /* largest gap between consecutive primes in range */
  uint64_t max_gap_lo;      /* lower prime of the first maximal gap */
  uint64_t mod4[2];         /* [0] = #p = 1 mod 4, [1] = #p = 3 mod 4: pi(x;4,1), pi(x;4,3) (:682) */
  uint64_t modq[VOSS_MODQ_SLOTS]; /* counts by (q, p mod q), q in VOSS_Q_LIST, q-major */
  uint64_t modq_gap[VOSS_MODQ_ROWS][VOSS_MODQ_MAX_GAP]; /* [row][gap] (:758-771) */
  uint64_t large_total;     /* large gaps found (may exceed the caller's capacity) */
  uint64_t gap_hist[VOSS_MAX_GAP]; /* gaps_total[g] (:403,583,634-635) */
} voss_range_stats;

/* Per-interval statistics of a batched or served interval query. */
typedef struct voss_interval_stats {
  uint64_t lo, hi;          /* [lo, hi) */
  uint64_t prime_count;
  uint64_t first_prime, last_prime;   /* 0 if none */
  uint64_t max_gap, max_gap_lo;       /* 0 if fewer than two primes */
  uint64_t gap_overflow;              /* gaps >= 2*VOSS_IHIST (none exist below 2^64) */
  uint64_t gap_hist[VOSS_IHIST];      /* bin g/2 = #gaps of length g; bin 0 = #gaps of length 1 */
} voss_interval_stats;

/* Sieve tuning; zero fields take the library's defaults. */
typedef struct voss_tuning {
  uint32_t block_threads;   /* 512 or 1024 */
  uint32_t chunk_words;     /* odd; a tile is block_threads * chunk_words 32-bit words */
  uint32_t ctas_per_sm;     /* resident tiles per SM */
  uint32_t coop_div;        /* primes p < tile_bytes/coop_div are cleared warp-cooperatively */
  uint32_t mult_factor;     /* primes p >= mult_factor*tile_bytes use the multiples walk */
  uint32_t medium_mode;     /* other primes: 0 = a thread per prime, 1 = a lane per (prime, residue) */
  uint32_t walk_sixteenths; /* mode 0: primes p >= walk_sixteenths*tile_bytes/16 walk their coprime
                               multiples instead of 8 residue progressions (>= 16*mult_factor: never) */
  uint32_t mr_route;        /* voss_sieve_intervals: an interval whose base primes >= mult_factor*tile_bytes
                               outnumber mr_route times its length is tested by Miller-Rabin instead of
                               sieved (0 = default 50; 0xFFFFFFFF = never) */
} voss_tuning;

typedef struct voss_ctx voss_ctx;

/* ---- library / context ---------------------------------------------------- */
VOSS_API const char* voss_version(void);
VOSS_API const char* voss_last_error(void);
VOSS_API int voss_device_count(int* count);

/* Create a context on `device` able to sieve up to hi = max_hi: builds the base primes
 * 7 <= p <= isqrt(max_hi - 1) and keeps them resident on the device.
 * Replaces generate_base_primes + modinv caching (src/voss_v7_live.cu:96-118,357-360,427-431). */
VOSS_API int voss_ctx_create(int device, uint64_t max_hi, voss_ctx** out);
VOSS_API void voss_ctx_destroy(voss_ctx* ctx);
VOSS_API int voss_ctx_info(const voss_ctx* ctx, uint64_t* max_hi, uint64_t* n_base_primes,
                           int* sm_count);
VOSS_API int voss_ctx_set_tuning(voss_ctx* ctx, const voss_tuning* t);
VOSS_API int voss_ctx_get_tuning(const voss_ctx* ctx, voss_tuning* t);

/* ---- single-range sieve + statistics -------------------------------------- */
/* Sieve [lo, hi) on the device and fill `stats`; the large gaps (gap >= 500 or merit >= 10,
 * merit computed only for gap > 100: src/voss_v7_live.cu:289-299) go to `large`, up to
 * large_cap entries, in ascending position order; *large_written receives the count written.
 * Replaces the segment loop of voss_v7_live main() (:434-626) together with the
 * accumulation of its epilogue (:634-635,682); the artifacts are written by
 * voss_write_artifacts.  seg_num is used in REF_COMPAT mode only (must be a multiple of 30). */
VOSS_API int voss_sieve_range(voss_ctx* ctx, uint64_t lo, uint64_t hi, uint32_t flags,
                              uint64_t seg_num, voss_range_stats* stats,
                              voss_large_gap* large, uint64_t large_cap,
                              uint64_t* large_written);

/* Device-resident form of voss_sieve_range for timing: runs the same kernels on the
 * context's stream (`stream` = cudaStream_t or NULL for the context's own) and leaves the
 * results in device memory; voss_fetch_range copies them out and finishes the statistics. */
VOSS_API int voss_sieve_range_device(voss_ctx* ctx, uint64_t lo, uint64_t hi, uint32_t flags,
                                     uint64_t seg_num, void* stream);
VOSS_API int voss_fetch_range(voss_ctx* ctx, voss_range_stats* stats, voss_large_gap* large,
                              uint64_t large_cap, uint64_t* large_written);

/* Write the primes of [lo, hi) in ascending order to out[0..cap); *count receives the
 * number of primes in range (out holds min(count, cap) of them).  No counterpart in the
 * reference beyond its internal positions[] array (src/voss_v7_live.cu:145-179,522-523). */
VOSS_API int voss_primes_range(voss_ctx* ctx, uint64_t lo, uint64_t hi, uint64_t* out,
                               uint64_t cap, uint64_t* count);

/* Every gap g >= min_gap (min_gap >= 3) between consecutive primes of [lo, hi), as
 * (p_after, g, merit = g / log(p_before)) in ascending position order: the input list of the
 * interior-composite proofs.  *count receives the number found; out holds min(count, cap).
 * The reference's large-gap rule is fixed (gap >= 500 or merit >= 10, src/voss_v7_live.cu:291);
 * this entry point has no counterpart there. */
VOSS_API int voss_gaps_at_least(voss_ctx* ctx, uint64_t lo, uint64_t hi, uint32_t min_gap,
                                voss_large_gap* out, uint64_t cap, uint64_t* count);

/* ---- batched intervals ----------------------------------------------------- */
/* Sieve n independent intervals [lo[i], hi[i]) in one persistent launch over an
 * (interval, tile) work queue and fill out[i].  The reference has no interval API; each
 * result equals a one-interval call on the same range. */
VOSS_API int voss_sieve_intervals(voss_ctx* ctx, const uint64_t* lo, const uint64_t* hi,
                                  uint32_t n, voss_interval_stats* out);

/* ---- Miller-Rabin and gap proofs -------------------------------------------- */
/* is_prime[i] = is_prime_u64(n[i]) of src/verify_cpp.cpp:38-57 (12 bases 2..37). */
VOSS_API int voss_mr_verify(voss_ctx* ctx, const uint64_t* n, uint64_t count, uint8_t* is_prime);
/* Device pointers; `stream` as for voss_sieve_range_device. */
VOSS_API int voss_mr_verify_device(voss_ctx* ctx, const uint64_t* d_n, uint64_t count,
                                   uint8_t* d_is_prime, void* stream);
/* The same verdicts as voss_mr_verify_device, for callers that cannot allocate device memory
 * during the call: processes whose device memory is already reserved by another allocator (a
 * framework's caching allocator or a memory pool), and service request paths where
 * cudaMalloc/cudaFree would synchronize the device.  No counterpart in the reference.
 * It takes no context and allocates nothing: its scratch is a fixed array inside libvoss.so
 * (16 MiB, held on every device that loads the library until exit), so
 *   - count may not exceed 4194304 (1 << 22) per call; larger counts return VOSS_ERR_ARG;
 *   - every call shares that array: calls that overlap on the GPU (different streams, or
 *     different host threads on one device) race; order them on one stream;
 *   - the first call on a device sets up (looks up the array's device address and uploads the
 *     Miller-Rabin constant tables) on the calling thread's current device; make that first
 *     call before any stream capture.
 * d_n and d_is_prime are device pointers on the current device; `stream` is a cudaStream_t or
 * NULL for the legacy default stream.  The call is asynchronous on `stream`. */
VOSS_API int voss_mr_verify_noalloc(const uint64_t* d_n, uint64_t count, uint8_t* d_is_prime,
                                    void* stream);
/* ok[i] = verify_gap(p_after[i], gap[i]) of src/verify_cpp.cpp:59-93: both ends prime and
 * every interior integer marked by the reference's interval sieve. */
VOSS_API int voss_prove_gaps(voss_ctx* ctx, const uint64_t* p_after, const int32_t* gap,
                             uint64_t count, uint8_t* ok);

/* SHA-256 of count messages at once (the digest step of the gap certificates,
 * scripts/generate_certificates.py:105-108, which hashes "VOSS|p_before|p_after|gap|merit:.6f"
 * with hashlib one string at a time).  Message i is data[offsets[i] .. offsets[i+1]);
 * offsets has count + 1 entries, offsets[0] = 0, non-decreasing.  digests receives 32 bytes
 * per message (the FIPS 180-4 digest, big-endian words).  Host buffers. */
VOSS_API int voss_sha256_batch(voss_ctx* ctx, const uint8_t* data, const uint64_t* offsets,
                               uint64_t count, uint8_t* digests);

/* ---- artifacts --------------------------------------------------------------- */
/* Write gap_histogram.csv, hl_trend.csv, modq_counts.csv, modq_gap_hist.csv,
 * chebyshev.csv and large_gaps.csv into `dir` in the byte format of
 * src/voss_v7_live.cu:707-827 (large gaps sorted by merit, descending, ties by position).
 * `stats` must come from a REF_COMPAT call with lo = 1. */
VOSS_API int voss_write_artifacts(const voss_range_stats* stats, const voss_large_gap* large,
                                  uint64_t n_large, const char* dir);

/* Combine the statistics of adjacent ranges parts[0..n) (parts[i].hi == parts[i+1].lo, same
 * flags and seg_num) into one, adding the gaps between neighbouring parts: the host half of
 * a range sharded across GPUs.  large_* describe the concatenated large-gap lists; the
 * boundary gaps that qualify are appended to large[] up to large_cap. */
VOSS_API int voss_stats_merge(const voss_range_stats* parts, uint32_t n, voss_range_stats* out,
                              voss_large_gap* large, uint64_t n_large, uint64_t large_cap,
                              uint64_t* large_written);

/* ---- segment-level features: gap sequence, checkpoint / resume ------------------- */
/* The sampled gap sequence of gap_sequence.csv (src/voss_v7_live.cu:234-253,526-547): for each
 * segment s of [1, n] of length seg_num, per_seg = seq_size / NUM_SEG consecutive gaps starting
 * at the middle prime (by count) of the segment's primes >= 7, at indices s*per_seg ...;
 * gap[i] = p_next - p, p_lo[i] = p; unwritten entries are 0 (the reference leaves them
 * uninitialised).  *written receives the number of gaps written. */
VOSS_API int voss_gap_sequence(voss_ctx* ctx, uint64_t n, uint64_t seg_num, uint64_t seq_size,
                               int32_t* gap, uint64_t* p_lo, uint64_t* written);
/* gap_sequence.csv "index,gap,p" rows for gap[i] > 0 (src/voss_v7_live.cu:786-803). */
VOSS_API int voss_write_gap_sequence(const int32_t* gap, const uint64_t* p_lo, uint64_t seq_size,
                                     const char* dir);

/* Statistics of one segment [lo, hi) into out/large: the unit of work of a checkpointed run. */
typedef int (*voss_segment_fn)(void* user, uint64_t lo, uint64_t hi, voss_range_stats* out,
                               voss_large_gap* large, uint64_t large_cap, uint64_t* large_written);
/* [1, n] segment by segment (segments of seg_num integers, a multiple of 30), merging each into
 * the running statistics; dir/checkpoint.bin is saved after the first, the last and every
 * ckpt_every-th segment (src/voss_v7_live.cu:599-602) and holds every accumulator, so a resumed
 * run equals an uninterrupted one; if dir/stop.txt exists at a save, it is removed and the call
 * returns VOSS_ERR_STOPPED (:603-620).  A valid checkpoint for the same (n, seg_num, flags) is
 * resumed from (*resumed_from = its next segment); the file is removed on success. */
VOSS_API int voss_run_checkpointed(voss_ctx* ctx, uint64_t n, uint64_t seg_num, uint32_t flags,
                                   uint32_t ckpt_every, const char* dir, voss_range_stats* out,
                                   voss_large_gap* large, uint64_t large_cap, uint64_t* large_written,
                                   uint64_t* resumed_from);
/* The same driver over any segment function (the device sieve in voss_run_checkpointed). */
VOSS_API int voss_run_checkpointed_fn(voss_segment_fn fn, void* user, uint64_t n, uint64_t seg_num,
                                      uint32_t flags, uint32_t ckpt_every, const char* dir,
                                      voss_range_stats* out, voss_large_gap* large, uint64_t large_cap,
                                      uint64_t* large_written, uint64_t* resumed_from);

/* ---- serving: continuous batching ------------------------------------------------ */
/* A request server over one context.  Client threads submit interval-sieve + gap-statistics
 * requests and Miller-Rabin batches; a scheduler thread launches the pending requests, in
 * arrival order, as one batch on whichever of `slots` streams is free (one persistent tile
 * launch for all the batch's intervals, one Miller-Rabin launch for all its candidates), so
 * requests that arrive while others run are admitted as slots free up and batches overlap on
 * the device.  Each slot's device memory and pinned staging is sized at creation from the
 * config (requests, tiles = bitmap memory, candidates); serving then allocates nothing on the
 * device.  Every wait is bounded.  The server is thread-safe; while it runs, the context's own
 * entry points may be used only from one other thread.  No counterpart in the reference. */
typedef struct voss_server voss_server;
typedef struct voss_server_config {
  uint32_t slots;                 /* batches in flight (streams); default 4 */
  uint32_t max_batch_requests;    /* interval requests per batch; default 1024 */
  uint32_t max_batch_tiles;       /* tiles per batch (one tile = 6.02e6 integers by default); default 65536 */
  uint32_t fail_every_n_batches;  /* testing: fail every n-th batch on the host (0 = never) */
  uint64_t max_batch_candidates;  /* Miller-Rabin candidates per batch; default 1 << 22 */
  uint64_t max_batch_bitmap_bytes; /* large-prime bitmap per slot (bytes = integers/30); default 1 GiB */
  uint64_t reserved[1];
} voss_server_config;
typedef struct voss_server_stats {
  uint64_t batches, completed, failed, pending, kernel_launches;
  uint32_t max_inflight_batches;
  uint32_t reserved0;
  double mean_batch_requests;
} voss_server_stats;

VOSS_API int voss_server_create(voss_ctx* ctx, const voss_server_config* cfg, voss_server** out);
/* Drains queued and running requests, then stops the scheduler and frees the slots. */
VOSS_API void voss_server_destroy(voss_server* srv);
/* Queue [lo, hi); the answer is a voss_interval_stats equal to voss_sieve_intervals on it alone. */
VOSS_API int voss_server_submit_interval(voss_server* srv, uint64_t lo, uint64_t hi, uint64_t* ticket);
/* Queue Miller-Rabin verdicts for n[0..count) (copied at submission, by up to 8 host threads for
 * large batches; VOSS_ERR_NOMEM when the host copy cannot be allocated). */
VOSS_API int voss_server_submit_mr(voss_server* srv, const uint64_t* n, uint64_t count, uint64_t* ticket);
/* VOSS_OK once the request finished, VOSS_ERR_TIMEOUT after timeout_ms, or the request's error. */
VOSS_API int voss_server_wait(voss_server* srv, uint64_t ticket, uint32_t timeout_ms);
VOSS_API int voss_server_result_interval(voss_server* srv, uint64_t ticket, voss_interval_stats* out);
VOSS_API int voss_server_result_mr(voss_server* srv, uint64_t ticket, uint8_t* out, uint64_t count);
/* Seconds since server creation at submission, batch start and completion (-1 if not yet). */
VOSS_API int voss_server_request_times(voss_server* srv, uint64_t ticket, double* submit_s, double* start_s,
                                       double* done_s);
/* Forget a finished request (voss_request_free). */
VOSS_API int voss_server_release(voss_server* srv, uint64_t ticket);
VOSS_API int voss_server_get_stats(voss_server* srv, voss_server_stats* out);

/* ---- diagnostics --------------------------------------------------------------- */
/* Shared-memory read-modify-write bandwidth of this device (GB/s, 8 bytes per 32-bit
 * atomicAnd), measured by a bank-conflict-free kernel: the roofline denominator of the
 * shared-memory-bound sieve.  No counterpart in the reference. */
VOSS_API int voss_probe_smem_rmw(voss_ctx* ctx, double* gbs);
/* Montgomery products per second of this device (independent squaring chains, all lanes
 * active, no memory traffic), for moduli of 64 bits (full) and below 2^63 (small): the roofline
 * denominator of the Miller-Rabin kernels.  No counterpart in the reference. */
VOSS_API int voss_probe_mulmod(voss_ctx* ctx, double* full_per_s, double* small_per_s);
/* Device time (ms, CUDA events) of the last sieve launch on the context's events
 * (voss_sieve_range[_device], voss_sieve_intervals, voss_gaps_at_least, voss_primes_range):
 * sieve_ms from the launch's first device operation (descriptor copies, memsets) to the end of
 * the tile kernel, total_ms to the end of its last kernel. */
VOSS_API int voss_last_kernel_ms(const voss_ctx* ctx, double* sieve_ms, double* total_ms);
/* The same launch in three consecutive phases: prepass_ms = descriptor copies, memsets and the
 * large-prime pre-pass kernels; tile_ms = the tile kernel alone; tail_ms = the stitch, reduce and
 * (intervals) finalize kernels; kernels = how many kernels the launch ran. */
VOSS_API int voss_last_phase_ms(const voss_ctx* ctx, double* prepass_ms, double* tile_ms, double* tail_ms,
                                uint32_t* kernels);

#ifdef __cplusplus
}
#endif

#endif /* VOSS_H */

// voss_server.cpp — request server with continuous batching (voss_server_* in include/voss.h).
//
// The reference has no serving mode.  Requests (interval sieve + gap statistics, or a batch of
// Miller-Rabin candidates) are queued by any number of client threads.  One scheduler thread owns
// K "slots"; each slot is a CUDA stream with its own device workspace and pinned host staging,
// all sized at creation so that batches never allocate device or pinned memory (a Miller-Rabin
// request keeps a host copy of its candidates until it is released).  Whenever a slot is free and requests
// are pending, the scheduler takes the pending requests in arrival order until the slot's
// capacity (requests, tiles = bitmap memory, candidates) is reached and launches them as one
// batch: one persistent tile-kernel launch over all the batch's (interval, tile) work items,
// then one Miller-Rabin launch over all its candidates.  Requests that arrive while batches run
// are admitted into the next slot that frees up, so batches overlap on the device.  A slot's
// completion is an event recorded behind its last copy, which the scheduler polls while batches
// are in flight (it sleeps on a condition variable only when the server is idle); every wait is
// bounded.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "voss_host.h"

using namespace voss_host;
using voss::IntervalOut;
using voss::SieveArgs;

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { kPending = 1, kRunning = 2, kDone = 0 };

// Candidate payloads are copied by up to 8 host threads in parts of at least 1 MB: one thread
// copies at a fraction of the host's memory bandwidth, and a thread costs tens of microseconds.
constexpr size_t kCopyPart = 1u << 20;

struct Request {
  uint64_t id = 0;
  int kind = 0;  // 0: interval, 1: Miller-Rabin
  uint64_t lo = 0, hi = 0;
  uint32_t tiles = 0;
  std::unique_ptr<uint64_t[]> in;  // Miller-Rabin candidates (not zero-filled before the copy)
  uint64_t n_in = 0;
  std::vector<uint8_t> out;
  voss_interval_stats st;
  Clock::time_point t_submit, t_start, t_done;
  int state = kPending;
  int error = VOSS_OK;
};

struct Slot {
  cudaStream_t stream = nullptr;
  Workspace ws;
  LaunchEvents E;
  bool busy = false;
  bool ready = false;            // the batch's work (or its failed launch) is finished
  cudaEvent_t done = nullptr;    // recorded behind the batch's last copy
  std::vector<Request*> iv, mr;
  uint32_t n_iv = 0;
  uint64_t n_mr = 0;
  voss_interval_stats* h_istats = nullptr;
  uint64_t* h_mr_in = nullptr;
  uint8_t* h_mr_out = nullptr;
  uint32_t* h_ctr = nullptr;
  int launch_error = VOSS_OK;
  struct voss_server* owner = nullptr;
};

}  // namespace

struct voss_server {
  voss_ctx* ctx = nullptr;
  voss_server_config cfg{};
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::atomic<uint64_t> submitted{0};  // requests ever enqueued: the polling scheduler's wake-up
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread th;
  Clock::time_point t0;
  uint64_t batches = 0, completed = 0, failed = 0, batched_requests = 0;
  uint32_t inflight = 0, max_inflight = 0;
  uint64_t launches = 0;
};

namespace {

double secs(const voss_server* S, Clock::time_point t) {
  return std::chrono::duration<double>(t - S->t0).count();
}

uint32_t tiles_of(const voss_ctx* c, uint64_t lo, uint64_t hi) {
  const uint64_t a = lo < 7 ? 7 : lo;
  if (a >= hi) return 0;
  const uint64_t k0 = (a / 30) & ~3ull, kl = (hi - 1) / 30;
  const uint64_t words = (kl - k0) / 4 + 1;
  const uint64_t tw = (uint64_t)c->tune.block_threads * c->tune.chunk_words;
  const uint64_t t = (words + tw - 1) / tw;
  return t > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)t;
}

// Poll a busy slot's completion event: true once its work is done (or the query failed, which
// fails the batch).
bool slot_finished(Slot& sl) {
  const cudaError_t e = cudaEventQuery(sl.done);
  if (e == cudaErrorNotReady) return false;
  if (e != cudaSuccess) {
    cudaGetLastError();
    sl.launch_error = fail(VOSS_ERR_CUDA, "batch completion query failed: %s", cudaGetErrorString(e));
  }
  return true;
}

// Queue one batch on a free slot (called without the server lock; the batch lists are owned by
// the scheduler thread until completion).
int launch_batch(voss_server* S, Slot& sl) {
  NvtxRange nvtx_("server batch launch");
  voss_ctx* c = S->ctx;
  cudaStream_t s = sl.stream;
  sl.n_iv = (uint32_t)sl.iv.size();
  if (S->cfg.fail_every_n_batches && (S->batches % S->cfg.fail_every_n_batches) == S->cfg.fail_every_n_batches - 1)
    return fail(VOSS_ERR_CUDA, "injected batch failure (fail_every_n_batches)");
  if (sl.n_iv) {
    std::vector<uint64_t> lo(sl.n_iv), hi(sl.n_iv);
    for (uint32_t i = 0; i < sl.n_iv; ++i) {
      lo[i] = sl.iv[i]->lo;
      hi[i] = sl.iv[i]->hi;
    }
    // short intervals at high starts by Miller-Rabin, within the slot's candidate buffers (the
    // batch's own Miller-Rabin requests reuse them later on the same stream)
    IntervalRoute R;
    route_intervals(c, lo.data(), hi.data(), sl.n_iv, S->cfg.max_batch_candidates, &R);
    uint32_t kernels = 0;
    int rc = launch_routed(c, sl.ws, sl.E, R, sl.n_iv, s, &kernels);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(sl.h_istats, sl.ws.istats.p, sizeof(voss_interval_stats) * sl.n_iv,
                             cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(sl.h_ctr, sl.ws.counters.p, sizeof(uint32_t) * kCtrWords, cudaMemcpyDeviceToHost, s));
    S->launches += kernels;
  } else {
    std::memset(sl.h_ctr, 0, sizeof(uint32_t) * kCtrWords);
  }
  // the batch's candidates into the slot's pinned staging, split over host threads
  sl.n_mr = 0;
  std::vector<CopySeg> segs;
  segs.reserve(sl.mr.size());
  for (Request* r : sl.mr) {
    segs.push_back(CopySeg{r->in.get(), r->n_in * 8});
    sl.n_mr += r->n_in;
  }
  parallel_gather(sl.h_mr_in, segs.data(), segs.size(), kCopyPart);
  if (sl.n_mr) {
    CUDA_TRY(cudaMemcpyAsync(sl.ws.mr_in.p, sl.h_mr_in, sl.n_mr * 8, cudaMemcpyHostToDevice, s));
    uint32_t* work = sl.ws.mr_work.as<uint32_t>();
    if (voss::launch_mr(sl.ws.mr_in.as<uint64_t>(), sl.n_mr, sl.ws.mr_out.as<uint8_t>(), work + 8, work, s,
                        c->sm_count))
      return fail(VOSS_ERR_CUDA, "Miller-Rabin launch failed");
    CUDA_TRY(cudaMemcpyAsync(sl.h_mr_out, sl.ws.mr_out.p, sl.n_mr, cudaMemcpyDeviceToHost, s));
    S->launches += 2;
  }
  CUDA_TRY(cudaEventRecord(sl.done, s));
  return VOSS_OK;
}

// Deliver a finished slot's results (called with the server lock held).
void complete_slot(voss_server* S, Slot& sl) {
  NvtxRange nvtx_("server batch complete");
  const auto now = Clock::now();
  int err = sl.launch_error;
  if (!err && sl.n_iv) err = check_device_error(sl.h_ctr);
  for (uint32_t i = 0; i < sl.iv.size(); ++i) {
    Request* r = sl.iv[i];
    if (!err) {
      std::memcpy(&r->st, &sl.h_istats[i], sizeof(voss_interval_stats));
      add_small_primes(r->st, r->lo, r->hi);
    }
    r->error = err;
    r->state = kDone;
    r->t_done = now;
  }
  uint64_t off = 0;
  for (Request* r : sl.mr) {
    if (!err) {
      r->out.resize(r->n_in);
      std::memcpy(r->out.data(), sl.h_mr_out + off, r->n_in);
    }
    off += r->n_in;
    r->error = err;
    r->state = kDone;
    r->t_done = now;
  }
  const uint64_t nreq = sl.iv.size() + sl.mr.size();
  S->completed += err ? 0 : nreq;
  S->failed += err ? nreq : 0;
  sl.iv.clear();
  sl.mr.clear();
  sl.busy = false;
  sl.ready = false;
  sl.launch_error = VOSS_OK;
  S->inflight--;
  S->cv_done.notify_all();
}

// Take pending requests in arrival order while they fit the slot (called with the lock held).
bool form_batch(voss_server* S, Slot& sl) {
  uint32_t tiles = 0;
  uint64_t cand = 0;
  const auto now = Clock::now();
  while (!S->pending.empty()) {
    Request* r = S->pending.front();
    if (r->kind == 0) {
      if (sl.iv.size() >= S->cfg.max_batch_requests || tiles + r->tiles > S->cfg.max_batch_tiles) break;
      tiles += r->tiles;
      sl.iv.push_back(r);
    } else {
      if (cand + r->n_in > S->cfg.max_batch_candidates) break;
      cand += r->n_in;
      sl.mr.push_back(r);
    }
    r->state = kRunning;
    r->t_start = now;
    S->pending.pop_front();
  }
  return !sl.iv.empty() || !sl.mr.empty();
}

void scheduler(voss_server* S) {
  cudaSetDevice(S->ctx->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    for (auto& up : S->slots)
      if (up->busy && (up->ready || slot_finished(*up))) complete_slot(S, *up);
    if (S->stop && S->pending.empty() && S->inflight == 0) break;
    bool launched = false;
    for (auto& up : S->slots) {
      Slot& sl = *up;
      if (sl.busy || S->pending.empty()) continue;
      if (!form_batch(S, sl)) continue;
      sl.busy = true;
      S->inflight++;
      if (S->inflight > S->max_inflight) S->max_inflight = S->inflight;
      S->batches++;
      S->batched_requests += sl.iv.size() + sl.mr.size();
      lk.unlock();
      const int rc = launch_batch(S, sl);
      lk.lock();
      if (rc != VOSS_OK) {  // nothing (more) will complete on this slot: drain it, then fail the batch
        lk.unlock();
        cudaStreamSynchronize(sl.stream);
        lk.lock();
        sl.launch_error = rc;
        sl.ready = true;
        complete_slot(S, sl);
      }
      launched = true;
    }
    if (launched) continue;
    if (S->inflight > 0) {
      // batches on the GPU: poll their completion events (and new submissions) instead of
      // sleeping, so a finished batch is delivered within microseconds rather than after a
      // driver callback thread and a condition-variable wake-up
      const uint64_t seen = S->submitted.load(std::memory_order_acquire);
      lk.unlock();
      for (;;) {
        bool any = false;
        for (auto& up : S->slots)
          if (up->busy && !up->ready && cudaEventQuery(up->done) != cudaErrorNotReady) any = true;
        if (any || S->submitted.load(std::memory_order_acquire) != seen) break;
        std::this_thread::yield();
      }
      lk.lock();
      continue;
    }
    // idle: woken by submissions; the timeout is a safety net
    S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
  }
}

Slot* make_slot(voss_server* S, int* rc) {
  auto sl = new Slot();
  sl->owner = S;
  const voss_server_config& C = S->cfg;
  voss_ctx* c = S->ctx;
  const uint64_t nreq = C.max_batch_requests ? C.max_batch_requests : 1;
  auto bad = [&](int code) {
    *rc = code;
    return sl;
  };
  if (cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&sl->E.ev0) != cudaSuccess || cudaEventCreate(&sl->E.ev1) != cudaSuccess ||
      cudaEventCreate(&sl->E.ev2) != cudaSuccess ||
      cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming) != cudaSuccess)
    return bad(fail(VOSS_ERR_CUDA, "server slot stream/event creation failed"));
  Workspace& W = sl->ws;
  int e;
  if ((e = W.iv.ensure(sizeof(voss::IntervalDev) * nreq)) || (e = W.partials.ensure(sizeof(voss::TilePartial) * C.max_batch_tiles)) ||
      (e = W.tile_iv.ensure(sizeof(uint32_t) * C.max_batch_tiles)) ||
      (e = W.acc.ensure(sizeof(unsigned long long) * voss::kAccStride * nreq)) ||
      (e = W.out.ensure(sizeof(IntervalOut) * nreq)) || (e = W.counters.ensure(sizeof(uint32_t) * kCtrWords)) ||
      (e = W.over.ensure(sizeof(voss::OverflowGap) * kOverCap)) || (e = W.large.ensure(sizeof(voss::LargeGapDev))) ||
      (e = W.large_iv.ensure(sizeof(uint32_t))) || (e = W.istats.ensure(sizeof(voss_interval_stats) * nreq)) ||
      (e = W.mr_in.ensure(8 * (C.max_batch_candidates + 1))) || (e = W.mr_out.ensure(C.max_batch_candidates + 1)) ||
      (e = W.mr_work.ensure(4 * (C.max_batch_candidates + 8))))
    return bad(e);
  // the large-prime pre-pass bitmap: fixed size, never grown while serving
  W.gbm_budget = C.max_batch_bitmap_bytes;
  W.gbm_fixed = true;
  if (W.gbm_budget && ((e = W.gbm.ensure(W.gbm_budget)) || (e = W.scat.ensure(sizeof(voss::IntervalScatter) * nreq))))
    return bad(e);
  if ((e = W.sh_iv.ensure(sizeof(voss::ShortInterval) * nreq)) || (e = W.sh_map.ensure(sizeof(uint32_t) * nreq)))
    return bad(e);
  if (cudaMallocHost(&sl->h_istats, sizeof(voss_interval_stats) * nreq) != cudaSuccess ||
      cudaMallocHost(&sl->h_mr_in, 8 * (C.max_batch_candidates + 1)) != cudaSuccess ||
      cudaMallocHost(&sl->h_mr_out, C.max_batch_candidates + 1) != cudaSuccess ||
      cudaMallocHost(&sl->h_ctr, sizeof(uint32_t) * kCtrWords) != cudaSuccess)
    return bad(fail(VOSS_ERR_NOMEM, "pinned host staging allocation failed"));
  (void)c;
  *rc = VOSS_OK;
  return sl;
}

void free_slot(Slot* sl) {
  if (!sl) return;
  if (sl->stream) cudaStreamSynchronize(sl->stream);
  if (sl->h_istats) cudaFreeHost(sl->h_istats);
  if (sl->h_mr_in) cudaFreeHost(sl->h_mr_in);
  if (sl->h_mr_out) cudaFreeHost(sl->h_mr_out);
  if (sl->h_ctr) cudaFreeHost(sl->h_ctr);
  if (sl->E.ev0) cudaEventDestroy(sl->E.ev0);
  if (sl->E.ev1) cudaEventDestroy(sl->E.ev1);
  if (sl->E.ev2) cudaEventDestroy(sl->E.ev2);
  if (sl->done) cudaEventDestroy(sl->done);
  if (sl->stream) cudaStreamDestroy(sl->stream);
  delete sl;
}

Request* find(voss_server* S, uint64_t ticket) {
  auto it = S->reqs.find(ticket);
  return it == S->reqs.end() ? nullptr : it->second.get();
}

uint64_t enqueue(voss_server* S, std::unique_ptr<Request> r) {
  Request* raw = r.get();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    raw->id = S->next_id++;
    raw->t_submit = Clock::now();
    S->reqs.emplace(raw->id, std::move(r));
    S->pending.push_back(raw);
    S->submitted.fetch_add(1, std::memory_order_release);
  }
  S->cv_work.notify_one();
  return raw->id;
}

}  // namespace

extern "C" {

VOSS_API int voss_server_create(voss_ctx* ctx, const voss_server_config* cfg, voss_server** out) {
  if (!ctx || !out) return fail(VOSS_ERR_ARG, "NULL argument");
  *out = nullptr;
  cudaSetDevice(ctx->device);
  auto S = std::make_unique<voss_server>();
  S->ctx = ctx;
  if (cfg) S->cfg = *cfg;
  voss_server_config& C = S->cfg;
  if (!C.slots) C.slots = 4;
  if (!C.max_batch_requests) C.max_batch_requests = 1024;
  if (!C.max_batch_tiles) C.max_batch_tiles = 1u << 16;
  if (!C.max_batch_candidates) C.max_batch_candidates = 1ull << 22;
  if (!C.max_batch_bitmap_bytes) C.max_batch_bitmap_bytes = 1ull << 30;
  if (C.slots > 64) return fail(VOSS_ERR_ARG, "at most 64 slots");
  if (C.max_batch_candidates > 0xFFFFFFF0ull) return fail(VOSS_ERR_ARG, "max_batch_candidates too large");
  for (uint32_t i = 0; i < C.slots; ++i) {
    int rc = VOSS_OK;
    Slot* sl = make_slot(S.get(), &rc);
    S->slots.emplace_back(sl);
    if (rc != VOSS_OK) {
      for (auto& up : S->slots) free_slot(up.release());
      return rc;
    }
  }
  S->t0 = Clock::now();
  S->th = std::thread(scheduler, S.get());
  *out = S.release();
  return VOSS_OK;
}

VOSS_API void voss_server_destroy(voss_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->th.joinable()) S->th.join();
  for (auto& up : S->slots) free_slot(up.release());
  delete S;
}

VOSS_API int voss_server_submit_interval(voss_server* S, uint64_t lo, uint64_t hi, uint64_t* ticket) {
  if (!S || !ticket) return fail(VOSS_ERR_ARG, "NULL argument");
  if (hi < lo) return fail(VOSS_ERR_ARG, "hi < lo");
  if (hi > S->ctx->max_hi) return fail(VOSS_ERR_RANGE, "hi exceeds the context limit");
  const uint32_t t = tiles_of(S->ctx, lo, hi);
  if (t > S->cfg.max_batch_tiles) return fail(VOSS_ERR_RANGE, "interval needs %u tiles, above the slot capacity %u", t, S->cfg.max_batch_tiles);
  auto r = std::make_unique<Request>();
  r->kind = 0;
  r->lo = lo;
  r->hi = hi;
  r->tiles = t;
  std::memset(&r->st, 0, sizeof(r->st));
  *ticket = enqueue(S, std::move(r));
  return VOSS_OK;
}

VOSS_API int voss_server_submit_mr(voss_server* S, const uint64_t* n, uint64_t count, uint64_t* ticket) {
  if (!S || !ticket || (count && !n)) return fail(VOSS_ERR_ARG, "NULL argument");
  if (count > S->cfg.max_batch_candidates)
    return fail(VOSS_ERR_RANGE, "%llu candidates exceed the slot capacity %llu", (unsigned long long)count,
                (unsigned long long)S->cfg.max_batch_candidates);
  auto r = std::make_unique<Request>();
  r->kind = 1;
  r->n_in = count;
  if (count) {
    r->in.reset(new (std::nothrow) uint64_t[count]);
    if (!r->in) return fail(VOSS_ERR_NOMEM, "no host memory for %llu candidates", (unsigned long long)count);
    parallel_copy(r->in.get(), n, count * 8, kCopyPart);
  }
  *ticket = enqueue(S, std::move(r));
  return VOSS_OK;
}

VOSS_API int voss_server_wait(voss_server* S, uint64_t ticket, uint32_t timeout_ms) {
  if (!S) return fail(VOSS_ERR_ARG, "NULL argument");
  std::unique_lock<std::mutex> lk(S->mu);
  Request* r = find(S, ticket);
  if (!r) return fail(VOSS_ERR_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  const bool done = S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->state == kDone; });
  if (!done) return fail(VOSS_ERR_TIMEOUT, "request %llu not finished after %u ms", (unsigned long long)ticket, timeout_ms);
  if (r->error) return fail(r->error, "request %llu failed", (unsigned long long)ticket);
  return VOSS_OK;
}

VOSS_API int voss_server_result_interval(voss_server* S, uint64_t ticket, voss_interval_stats* out) {
  if (!S || !out) return fail(VOSS_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  Request* r = find(S, ticket);
  if (!r || r->kind != 0) return fail(VOSS_ERR_ARG, "ticket %llu is not an interval request", (unsigned long long)ticket);
  if (r->state != kDone) return fail(VOSS_ERR_STATE, "request %llu not finished", (unsigned long long)ticket);
  if (r->error) return fail(r->error, "request %llu failed", (unsigned long long)ticket);
  std::memcpy(out, &r->st, sizeof(*out));
  return VOSS_OK;
}

VOSS_API int voss_server_result_mr(voss_server* S, uint64_t ticket, uint8_t* out, uint64_t count) {
  if (!S || (count && !out)) return fail(VOSS_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  Request* r = find(S, ticket);
  if (!r || r->kind != 1) return fail(VOSS_ERR_ARG, "ticket %llu is not a Miller-Rabin request", (unsigned long long)ticket);
  if (r->state != kDone) return fail(VOSS_ERR_STATE, "request %llu not finished", (unsigned long long)ticket);
  if (r->error) return fail(r->error, "request %llu failed", (unsigned long long)ticket);
  if (count != r->out.size()) return fail(VOSS_ERR_ARG, "count %llu differs from the request's %zu", (unsigned long long)count, r->out.size());
  std::memcpy(out, r->out.data(), count);
  return VOSS_OK;
}

VOSS_API int voss_server_request_times(voss_server* S, uint64_t ticket, double* submit_s, double* start_s, double* done_s) {
  if (!S) return fail(VOSS_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  Request* r = find(S, ticket);
  if (!r) return fail(VOSS_ERR_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  if (submit_s) *submit_s = secs(S, r->t_submit);
  if (start_s) *start_s = r->state == kPending ? -1.0 : secs(S, r->t_start);
  if (done_s) *done_s = r->state == kDone ? secs(S, r->t_done) : -1.0;
  return VOSS_OK;
}

VOSS_API int voss_server_release(voss_server* S, uint64_t ticket) {
  if (!S) return fail(VOSS_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return fail(VOSS_ERR_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  if (it->second->state != kDone) return fail(VOSS_ERR_STATE, "request %llu still queued or running", (unsigned long long)ticket);
  S->reqs.erase(it);
  return VOSS_OK;
}

VOSS_API int voss_server_get_stats(voss_server* S, voss_server_stats* out) {
  if (!S || !out) return fail(VOSS_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(out, 0, sizeof(*out));
  out->batches = S->batches;
  out->completed = S->completed;
  out->failed = S->failed;
  out->pending = S->pending.size();
  out->max_inflight_batches = S->max_inflight;
  out->mean_batch_requests = S->batches ? (double)S->batched_requests / (double)S->batches : 0.0;
  out->kernel_launches = S->launches;
  return VOSS_OK;
}

}  // extern "C"

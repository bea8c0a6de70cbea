// voss_driver.cpp — the reference program's segment-level features on top of the sieve:
// the sampled gap sequence (gap_sequence.csv) and checkpoint / resume with a stop file.
//
//  - voss_gap_sequence restates the sampler of src/voss_v7_live.cu:234-253 and :526-547: for
//    each segment s of length seg_num, per_seg = seq_size / NUM_SEG consecutive gaps starting at
//    the middle prime (by count) of the segment's primes >= 7, stored at index s * per_seg.
//  - voss_run_checkpointed runs [1, n] segment by segment like :434-626, merging every segment
//    into the running statistics (voss_stats_merge), saving a checkpoint on the reference's
//    schedule (first, last and every ckpt_every-th segment, :599-602) and stopping cleanly when
//    dir/stop.txt exists (:603-620).  Unlike the reference's CheckpointState (:44-54), the
//    checkpoint holds every accumulator (mod-q counts, per-residue gap histogram, large gaps),
//    so a resumed run produces exactly the artifacts of an uninterrupted one.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "voss_host.h"

using namespace voss_host;
using voss::TilePartial;

namespace {

// Pass 1: the tile plan of the wheel part [max(lo, 7), hi) and the prefix counts of its tiles'
// primes (prefix[t] = primes >= 7 before tile t).
int count_tiles(voss_ctx* c, uint64_t lo, uint64_t hi, RunPlan* P, std::vector<uint64_t>* prefix) {
  cudaStream_t s = c->stream;
  const uint64_t a = lo < 7 ? 7 : lo;
  prefix->assign(1, 0);
  P->iv.clear();
  P->n_tiles = 0;
  if (a >= hi) return VOSS_OK;
  int rc = plan_intervals(c, &a, &hi, 1, 0, P);
  if (rc) return rc;
  LaunchEvents E{c->ev0, c->ev1, c->ev2, c->evp};
  rc = launch_plan_ws(c, c->ws, E, *P, false, 0, false, s, 0, nullptr);
  if (rc) return rc;
  std::vector<TilePartial> parts(P->n_tiles);
  uint32_t ctr[kCtrWords];
  if (P->n_tiles)
    CUDA_TRY(cudaMemcpyAsync(parts.data(), c->ws.partials.p, sizeof(TilePartial) * P->n_tiles, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(ctr, c->ws.counters.p, sizeof(ctr), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if ((rc = check_device_error(ctr))) return rc;
  prefix->assign(P->n_tiles + 1, 0);
  for (uint32_t t = 0; t < P->n_tiles; ++t) (*prefix)[t + 1] = (*prefix)[t] + parts[t].count;
  return VOSS_OK;
}

// Pass 2: the primes >= 7 of plan P with rank in [r0, r0 + count), emitting only the tiles that
// hold them.
int emit_window(voss_ctx* c, const RunPlan& P, const std::vector<uint64_t>& prefix, uint64_t hi, uint64_t r0,
                uint64_t count, std::vector<uint64_t>* out) {
  cudaStream_t s = c->stream;
  out->clear();
  const uint64_t total = prefix.back();
  if (count == 0 || r0 >= total || P.n_tiles == 0) return VOSS_OK;
  const uint64_t r1 = std::min<uint64_t>(r0 + count, total);
  uint32_t t0 = 0, t1 = P.n_tiles - 1;
  while (prefix[t0 + 1] <= r0) ++t0;
  while (t1 > t0 && prefix[t1] >= r1) --t1;
  const uint64_t tw = (uint64_t)c->tune.block_threads * c->tune.chunk_words;
  const voss::IntervalDev& d = P.iv[0];
  const uint64_t sub_lo = t0 == 0 ? d.lo : 30ull * (d.k0 + 4ull * tw * t0);
  const uint64_t sub_hi = std::min<uint64_t>(hi, 30ull * (d.k0 + 4ull * tw * (t1 + 1)));
  RunPlan Q;
  int rc;
  if ((rc = plan_intervals(c, &sub_lo, &sub_hi, 1, 0, &Q))) return rc;
  std::vector<unsigned long long> offs(std::max<uint32_t>(1, Q.n_tiles));
  for (uint32_t t = 0; t < Q.n_tiles; ++t) offs[t] = prefix[t0 + t] - r0;  // wraps below r0: not written
  const uint64_t n = r1 - r0;
  if ((rc = c->ws.offsets.ensure(sizeof(unsigned long long) * offs.size())) ||
      (rc = c->ws.emit.ensure(sizeof(unsigned long long) * n)))
    return rc;
  CUDA_TRY(cudaMemcpyAsync(c->ws.offsets.p, offs.data(), sizeof(unsigned long long) * Q.n_tiles, cudaMemcpyHostToDevice, s));
  LaunchEvents E{c->ev0, c->ev1, c->ev2, c->evp};
  rc = launch_plan_ws(c, c->ws, E, Q, false, 0, true, s, 0, nullptr);
  if (rc) return rc;
  out->resize(n);
  uint32_t ctr[kCtrWords];
  CUDA_TRY(cudaMemcpyAsync(out->data(), c->ws.emit.p, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(ctr, c->ws.counters.p, sizeof(ctr), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return check_device_error(ctr);
}

// ---- checkpoint file ------------------------------------------------------------------
struct CkptHeader {
  char magic[8];
  uint32_t version;
  uint32_t flags;
  uint64_t n, seg_num, num_seg, next_segment, n_large, stats_bytes;
};
const char kMagic[8] = {'V', 'O', 'S', 'S', 'C', 'K', 'P', '1'};

int save_ckpt(const std::string& path, const CkptHeader& h, const voss_range_stats& st,
              const std::vector<voss_large_gap>& large) {
  NvtxRange nvtx_("checkpoint write");
  const std::string tmp = path + ".tmp";
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return fail(VOSS_ERR_IO, "cannot write %s", tmp.c_str());
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(&st, sizeof(st), 1, f) == 1 &&
            (large.empty() || std::fwrite(large.data(), sizeof(voss_large_gap), large.size(), f) == large.size());
  ok = (std::fclose(f) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) return fail(VOSS_ERR_IO, "cannot write %s", path.c_str());
  return VOSS_OK;
}

bool load_ckpt(const std::string& path, uint64_t n, uint64_t seg_num, uint32_t flags, CkptHeader* h,
               voss_range_stats* st, std::vector<voss_large_gap>* large) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  bool ok = std::fread(h, sizeof(*h), 1, f) == 1 && std::memcmp(h->magic, kMagic, 8) == 0 && h->version == 1 &&
            h->n == n && h->seg_num == seg_num && h->flags == flags && h->stats_bytes == sizeof(voss_range_stats) &&
            std::fread(st, sizeof(*st), 1, f) == 1;
  if (ok) {
    large->resize(h->n_large);
    ok = h->n_large == 0 || std::fread(large->data(), sizeof(voss_large_gap), h->n_large, f) == h->n_large;
  }
  std::fclose(f);
  return ok;
}

struct CtxSegment {
  voss_ctx* ctx;
  uint32_t flags;
  uint64_t seg_num;
};

int ctx_segment_fn(void* user, uint64_t lo, uint64_t hi, voss_range_stats* out, voss_large_gap* large,
                   uint64_t cap, uint64_t* written) {
  CtxSegment* cs = static_cast<CtxSegment*>(user);
  return voss_sieve_range(cs->ctx, lo, hi, cs->flags, cs->seg_num, out, large, cap, written);
}

}  // namespace

extern "C" {

VOSS_API int voss_gap_sequence(voss_ctx* c, uint64_t n, uint64_t seg_num, uint64_t seq_size, int32_t* gap,
                               uint64_t* p_lo, uint64_t* written) {
  NvtxRange nvtx_("voss_gap_sequence");
  if (!c || (seq_size && (!gap || !p_lo))) return fail(VOSS_ERR_ARG, "NULL argument");
  if (seg_num == 0 || seg_num % 30) return fail(VOSS_ERR_ARG, "seg_num must be a positive multiple of 30");
  if (n + 1 > c->max_hi) return fail(VOSS_ERR_RANGE, "n exceeds the context limit");
  cudaSetDevice(c->device);
  if (seq_size) {
    std::memset(gap, 0, sizeof(int32_t) * seq_size);
    std::memset(p_lo, 0, sizeof(uint64_t) * seq_size);
  }
  uint64_t w = 0;
  const uint64_t num_seg = (n + seg_num - 1) / seg_num;
  const uint64_t per_seg = num_seg ? seq_size / num_seg : 0;
  std::vector<uint64_t> pr;
  for (uint64_t s = 0; s < num_seg && per_seg > 0; ++s) {
    const uint64_t lo = s * seg_num + 1;
    const uint64_t hi = std::min<uint64_t>((s + 1) * seg_num, n) + 1;
    // pass 1 counts the segment's primes >= 7; the window is then [n_pos/2, n_pos/2 + sample_n]
    RunPlan P;
    std::vector<uint64_t> prefix;
    int rc = count_tiles(c, lo, hi, &P, &prefix);
    if (rc) return rc;
    const uint64_t n_pos = prefix.back();
    if (n_pos <= 1) continue;
    const uint64_t start = n_pos / 2;
    const uint64_t avail = n_pos - start - 1;
    const uint64_t sample_n = avail < per_seg ? avail : per_seg;
    if (sample_n <= 1) continue;
    const uint64_t offset = s * per_seg;
    if (offset + sample_n > seq_size) continue;
    rc = emit_window(c, P, prefix, hi, start, sample_n + 1, &pr);
    if (rc) return rc;
    if (pr.size() != sample_n + 1) return fail(VOSS_ERR_STATE, "gap sample window incomplete");
    for (uint64_t i = 0; i < sample_n; ++i) {
      gap[offset + i] = (int32_t)(pr[i + 1] - pr[i]);
      p_lo[offset + i] = pr[i];
    }
    w += sample_n;
  }
  if (written) *written = w;
  return VOSS_OK;
}

VOSS_API int voss_write_gap_sequence(const int32_t* gap, const uint64_t* p_lo, uint64_t seq_size, const char* dir) {
  if (!dir || (seq_size && (!gap || !p_lo))) return fail(VOSS_ERR_ARG, "NULL argument");
  const std::string path = std::string(dir) + "/gap_sequence.csv";
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) return fail(VOSS_ERR_IO, "cannot write %s", path.c_str());
  std::fprintf(f, "index,gap,p\n");  // src/voss_v7_live.cu:794-798
  for (uint64_t i = 0; i < seq_size; ++i)
    if (gap[i] > 0) std::fprintf(f, "%d,%d,%llu\n", (int)i, gap[i], (unsigned long long)p_lo[i]);
  std::fclose(f);
  return VOSS_OK;
}

VOSS_API int voss_run_checkpointed_fn(voss_segment_fn fn, void* user, uint64_t n, uint64_t seg_num, uint32_t flags,
                                      uint32_t ckpt_every, const char* dir, voss_range_stats* out,
                                      voss_large_gap* large, uint64_t large_cap, uint64_t* large_written,
                                      uint64_t* resumed_from) {
  NvtxRange nvtx_("voss_run_checkpointed_fn");
  if (!fn || !dir || !out) return fail(VOSS_ERR_ARG, "NULL argument");
  if (n < 1 || seg_num == 0 || seg_num % 30) return fail(VOSS_ERR_ARG, "need n >= 1 and seg_num a positive multiple of 30");
  if (!ckpt_every) ckpt_every = 5;
  const std::string dirs(dir);
  const std::string ck = dirs + "/checkpoint.bin", stop = dirs + "/stop.txt";
  const uint64_t num_seg = (n + seg_num - 1) / seg_num;
  std::vector<voss_range_stats> buf(3);  // running, segment, merged (too large for the stack)
  voss_range_stats& acc = buf[0];
  voss_range_stats& part = buf[1];
  voss_range_stats& merged = buf[2];
  std::vector<voss_large_gap> L;
  CkptHeader h;
  uint64_t next = 0;
  if (load_ckpt(ck, n, seg_num, flags, &h, &acc, &L)) {
    next = h.next_segment;
  } else {
    std::memset(&acc, 0, sizeof(acc));
    acc.lo = acc.hi = 1;
    acc.flags = flags;
    acc.seg_num = (flags & VOSS_FLAG_REF_COMPAT) ? seg_num : 0;
    L.clear();
  }
  if (resumed_from) *resumed_from = next;
  std::vector<voss_large_gap> seg_large;
  for (uint64_t s = next; s < num_seg; ++s) {
    const uint64_t lo = s * seg_num + 1;
    const uint64_t hi = std::min<uint64_t>((s + 1) * seg_num, n) + 1;
    uint64_t cap = 1u << 20, got = 0;
    for (;;) {
      seg_large.resize(cap);
      int rc = fn(user, lo, hi, &part, seg_large.data(), cap, &got);
      if (rc) return rc;
      if (part.large_total <= cap) break;
      cap = part.large_total;
    }
    const size_t base = L.size();
    L.insert(L.end(), seg_large.begin(), seg_large.begin() + (std::ptrdiff_t)got);
    L.resize(L.size() + 1);  // room for the seam gap
    std::vector<voss_range_stats> pair(2);
    pair[0] = acc;
    pair[1] = part;
    uint64_t nl = 0;
    int rc = voss_stats_merge(pair.data(), 2, &merged, L.data(), base + got, L.size(), &nl);
    if (rc) return rc;
    L.resize(nl);
    acc = merged;
    if (s == 0 || s == num_seg - 1 || (s + 1) % ckpt_every == 0) {
      std::memcpy(h.magic, kMagic, 8);
      h.version = 1;
      h.flags = flags;
      h.n = n;
      h.seg_num = seg_num;
      h.num_seg = num_seg;
      h.next_segment = s + 1;
      h.n_large = L.size();
      h.stats_bytes = sizeof(voss_range_stats);
      if ((rc = save_ckpt(ck, h, acc, L))) return rc;
      if (FILE* f = std::fopen(stop.c_str(), "r")) {
        std::fclose(f);
        std::remove(stop.c_str());
        return fail(VOSS_ERR_STOPPED, "stop file seen after segment %llu of %llu; checkpoint saved",
                    (unsigned long long)s + 1, (unsigned long long)num_seg);
      }
    }
  }
  std::remove(ck.c_str());
  std::memcpy(out, &acc, sizeof(acc));
  const uint64_t w = std::min<uint64_t>(L.size(), large ? large_cap : 0);
  if (w) std::memcpy(large, L.data(), sizeof(voss_large_gap) * w);
  if (large_written) *large_written = w;
  return VOSS_OK;
}

VOSS_API int voss_run_checkpointed(voss_ctx* ctx, uint64_t n, uint64_t seg_num, uint32_t flags, uint32_t ckpt_every,
                                   const char* dir, voss_range_stats* out, voss_large_gap* large, uint64_t large_cap,
                                   uint64_t* large_written, uint64_t* resumed_from) {
  if (!ctx) return fail(VOSS_ERR_ARG, "ctx is NULL");
  if (n + 1 > ctx->max_hi) return fail(VOSS_ERR_RANGE, "n exceeds the context limit");
  CtxSegment cs{ctx, flags, seg_num};
  return voss_run_checkpointed_fn(ctx_segment_fn, &cs, n, seg_num, flags, ckpt_every, dir, out, large, large_cap,
                                  large_written, resumed_from);
}

}  // extern "C"

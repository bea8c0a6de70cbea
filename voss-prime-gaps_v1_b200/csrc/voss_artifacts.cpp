// voss_artifacts.cpp — CSV artifacts and the merge of adjacent-range statistics.
//
// voss_write_artifacts writes the files of src/voss_v7_live.cu:707-827 byte for byte (same
// headers, row order, printf formats); voss_stats_merge is the host half of a range sharded
// over several GPUs: it sums the per-range statistics and adds the gap between neighbouring
// ranges with the rules the reference applies to every consecutive pair (:278-299, :559-562).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "voss.h"

namespace {

const int kW30[8] = {1, 7, 11, 13, 17, 19, 23, 29};

int set_err(int code, const char* msg);

struct File {
  FILE* f = nullptr;
  explicit File(const std::string& p) { f = std::fopen(p.c_str(), "w"); }
  ~File() {
    if (f) std::fclose(f);
  }
};

int row30(uint64_t p) {
  const int r = (int)(p % 30);
  for (int i = 0; i < 8; ++i)
    if (kW30[i] == r) return i;
  return -1;
}

}  // namespace

extern "C" const char* voss_last_error(void);
namespace voss_detail {
int set_error(int code, const char* msg);
}

namespace {
int set_err(int code, const char* msg) { return voss_detail::set_error(code, msg); }
}  // namespace

extern "C" {

VOSS_API int voss_write_artifacts(const voss_range_stats* st, const voss_large_gap* large,
                                  uint64_t n_large, const char* dir) {
  if (!st || !dir || (n_large && !large)) return set_err(VOSS_ERR_ARG, "NULL argument");
  const std::string d(dir);
  const long long N = (long long)(st->hi - 1);
  const int64_t* gaps = reinterpret_cast<const int64_t*>(st->gap_hist);

  {  // gap_histogram.csv (:707-711)
    File F(d + "/gap_histogram.csv");
    if (!F.f) return set_err(VOSS_ERR_IO, "cannot write gap_histogram.csv");
    std::fprintf(F.f, "gap,count\n");
    for (int g = 1; g < VOSS_MAX_GAP; g++)
      if (gaps[g] > 0) std::fprintf(F.f, "%d,%lld\n", g, (long long)gaps[g]);
  }
  {  // hl_trend.csv (:713-733): five fixed rows, then this N unless it is one of them
    File F(d + "/hl_trend.csv");
    if (!F.f) return set_err(VOSS_ERR_IO, "cannot write hl_trend.csv");
    static const long long kHlN[5] = {1000000000LL, 10000000000LL, 100000000000LL, 1000000000000LL,
                                      10000000000000LL};
    static const double kHlR[5] = {1.778300, 1.801800, 1.820800, 1.836600, 1.849700};
    std::fprintf(F.f, "N,P6_over_P2\n");
    bool already = false;
    for (int i = 0; i < 5; i++) {
      std::fprintf(F.f, "%lld,%.6f\n", kHlN[i], kHlR[i]);
      if (N == kHlN[i]) already = true;
    }
    if (!already) std::fprintf(F.f, "%lld,%.6f\n", N, (double)gaps[6] / (double)gaps[2]);
  }
  {  // modq_counts.csv (:735-751): q = 6 then q = 30, every residue
    File F(d + "/modq_counts.csv");
    if (!F.f) return set_err(VOSS_ERR_IO, "cannot write modq_counts.csv");
    std::fprintf(F.f, "q,a,count\n");
    const int qs[2] = {6, 30};
    const int offs[2] = {3 + 4 + 5, 3 + 4 + 5 + 6 + 7 + 8 + 11 + 12 + 13};
    for (int qi = 0; qi < 2; qi++)
      for (int a = 0; a < qs[qi]; a++)
        std::fprintf(F.f, "%d,%d,%llu\n", qs[qi], a, (unsigned long long)st->modq[offs[qi] + a]);
  }
  {  // modq_gap_hist.csv (:754-778)
    File F(d + "/modq_gap_hist.csv");
    if (!F.f) return set_err(VOSS_ERR_IO, "cannot write modq_gap_hist.csv");
    std::fprintf(F.f, "q,residue,gap,count\n");
    const int qv[2] = {6, 30}, qoff[2] = {0, 2}, nres[2] = {2, 8};
    const int res[2][8] = {{1, 5, 0, 0, 0, 0, 0, 0}, {1, 7, 11, 13, 17, 19, 23, 29}};
    for (int qi = 0; qi < 2; qi++)
      for (int ri = 0; ri < nres[qi]; ri++)
        for (int g = 1; g < VOSS_MODQ_MAX_GAP; g++) {
          const long long c = (long long)st->modq_gap[qoff[qi] + ri][g];
          if (c > 0) std::fprintf(F.f, "%d,%d,%d,%lld\n", qv[qi], res[qi][ri], g, c);
        }
  }
  {  // chebyshev.csv (:780-783)
    File F(d + "/chebyshev.csv");
    if (!F.f) return set_err(VOSS_ERR_IO, "cannot write chebyshev.csv");
    const unsigned long long p41 = st->mod4[0], p43 = st->mod4[1];
    std::fprintf(F.f, "N,pi_4_1,pi_4_3,difference\n");
    std::fprintf(F.f, "%lld,%llu,%llu,%lld\n", N, p41, p43, (long long)p43 - (long long)p41);
  }
  {  // large_gaps.csv (:805-827): by merit, descending (ties: ascending position)
    std::vector<voss_large_gap> v(large, large + n_large);
    std::sort(v.begin(), v.end(), [](const voss_large_gap& a, const voss_large_gap& b) {
      if (a.merit != b.merit) return a.merit > b.merit;
      return a.position < b.position;
    });
    File F(d + "/large_gaps.csv");
    if (!F.f) return set_err(VOSS_ERR_IO, "cannot write large_gaps.csv");
    std::fprintf(F.f, "position,gap,merit\n");
    for (const voss_large_gap& g : v)
      std::fprintf(F.f, "%llu,%d,%.6f\n", (unsigned long long)g.position, g.gap, (double)g.merit);
  }
  return VOSS_OK;
}

VOSS_API int voss_stats_merge(const voss_range_stats* parts, uint32_t n, voss_range_stats* out,
                              voss_large_gap* large, uint64_t n_large, uint64_t large_cap,
                              uint64_t* large_written) {
  if (!parts || !out || n == 0) return set_err(VOSS_ERR_ARG, "NULL argument or no parts");
  for (uint32_t i = 1; i < n; ++i) {
    if (parts[i].lo != parts[i - 1].hi) return set_err(VOSS_ERR_ARG, "parts are not adjacent");
    if (parts[i].flags != parts[0].flags || parts[i].seg_num != parts[0].seg_num)
      return set_err(VOSS_ERR_ARG, "parts have different modes");
  }
  const bool compat = (parts[0].flags & VOSS_FLAG_REF_COMPAT) != 0;
  const uint64_t seg = parts[0].seg_num;
  voss_range_stats* o = out;
  std::vector<voss_range_stats> tmp_buf(1);  // out may alias parts[0]; too large for the stack
  voss_range_stats& tmp = tmp_buf[0];
  std::memset(&tmp, 0, sizeof(tmp));
  tmp.lo = parts[0].lo;
  tmp.hi = parts[n - 1].hi;
  tmp.flags = parts[0].flags;
  tmp.seg_num = parts[0].seg_num;
  uint64_t nl = n_large;
  uint64_t extra = 0;
  uint64_t last = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const voss_range_stats& P = parts[i];
    if (P.prime_count == 0) continue;
    if (last) {  // the pair across the seam
      const uint64_t lo_p = last, hi_p = P.first_prime, g = hi_p - lo_p;
      if (g < VOSS_MAX_GAP) tmp.gap_hist[g]++;
      if (g > tmp.max_gap) {
        tmp.max_gap = g;
        tmp.max_gap_lo = lo_p;
      }
      const bool cross = compat && (lo_p - 1) / seg != (hi_p - 1) / seg;
      if (lo_p >= 7 && !cross) {
        if (g < VOSS_MODQ_MAX_GAP) {
          tmp.modq_gap[(lo_p % 6) == 1 ? 0 : 1][g]++;
          tmp.modq_gap[2 + row30(lo_p)][g]++;
        }
        double merit_d = 0.0;
        if (g > 100) merit_d = (double)g / std::log((double)lo_p);
        if ((g >= 500 || merit_d >= 10.0) && g < VOSS_MAX_GAP) {
          ++extra;
          if (large && nl < large_cap) large[nl++] = voss_large_gap{hi_p, (int32_t)g, (float)merit_d};
        }
      }
    } else {
      tmp.first_prime = P.first_prime;
    }
    if (P.max_gap > tmp.max_gap) {
      tmp.max_gap = P.max_gap;
      tmp.max_gap_lo = P.max_gap_lo;
    }
    tmp.prime_count += P.prime_count;
    tmp.mod4[0] += P.mod4[0];
    tmp.mod4[1] += P.mod4[1];
    for (int k = 0; k < VOSS_MODQ_SLOTS; ++k) tmp.modq[k] += P.modq[k];
    for (int r = 0; r < VOSS_MODQ_ROWS; ++r)
      for (int g = 0; g < VOSS_MODQ_MAX_GAP; ++g) tmp.modq_gap[r][g] += P.modq_gap[r][g];
    for (int g = 0; g < VOSS_MAX_GAP; ++g) tmp.gap_hist[g] += P.gap_hist[g];
    tmp.large_total += P.large_total;
    last = P.last_prime;
    tmp.last_prime = P.last_prime;
  }
  tmp.large_total += extra;
  std::memcpy(o, &tmp, sizeof(tmp));
  if (large_written) *large_written = nl;
  return VOSS_OK;
}

}  // extern "C"

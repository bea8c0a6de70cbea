// voss_verify — command-line drop-in for the reference's bin/verify_cpp, running the proofs on
// the GPU through libvoss.so.
//
// Same arguments and files as src/verify_cpp.cpp:112-276:
//   voss_verify [large_gaps.csv] [verification_details.csv] [verification_cache.csv]
// reads "position,gap,merit" rows (position = p_after), skips (p_after, gap) pairs already in
// the cache file ("p_after,gap" rows), proves the rest (both ends prime by the 12-base
// Miller-Rabin, interior composite: voss_prove_gaps), appends the verified pairs to the cache,
// writes "position,gap,merit,verified" rows in input order, and exits 1 if any gap failed.
// Its progress lines differ (there is no 30-second monitor thread); the files and the exit
// status are the reference's.
#include <chrono>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <unordered_set>
#include <vector>

#include "voss.h"

namespace {

struct PairKey {
  uint64_t p;
  int g;
  bool operator==(const PairKey& o) const { return p == o.p && g == o.g; }
};
struct PairKeyHash {
  size_t operator()(const PairKey& k) const {
    return std::hash<uint64_t>()(k.p) * 1000003u ^ std::hash<int>()(k.g);
  }
};

}  // namespace

int main(int argc, char** argv) {
  setvbuf(stdout, nullptr, _IONBF, 0);
  const char* input = argc > 1 ? argv[1] : "results/large_gaps.csv";
  const char* output = argc > 2 ? argv[2] : "results/verification_details.csv";
  const char* cache_path = argc > 3 ? argv[3] : "results/verification_cache.csv";
  const auto t0 = std::chrono::steady_clock::now();

  std::ifstream fin(input);
  if (!fin) {
    std::fprintf(stderr, "cannot open %s\n", input);
    return 1;
  }
  std::vector<uint64_t> p_after;
  std::vector<int32_t> gaps;
  std::vector<double> merits;
  std::string line;
  std::getline(fin, line);  // header
  while (std::getline(fin, line)) {
    if (line.empty()) continue;
    const size_t c1 = line.find(',');
    if (c1 == std::string::npos) continue;
    const size_t c2 = line.find(',', c1 + 1);
    p_after.push_back(std::stoull(line.substr(0, c1)));
    gaps.push_back(std::stoi(line.substr(c1 + 1, c2 == std::string::npos ? std::string::npos : c2 - c1 - 1)));
    merits.push_back(c2 != std::string::npos ? std::stod(line.substr(c2 + 1)) : 0.0);
  }
  const size_t n = p_after.size();
  std::printf("Read %zu gaps from %s\n", n, input);
  if (n == 0) return 1;

  std::unordered_set<PairKey, PairKeyHash> cache;
  {
    std::ifstream cf(cache_path);
    if (cf) {
      std::string cl;
      std::getline(cf, cl);
      while (std::getline(cf, cl)) {
        if (cl.empty()) continue;
        const size_t c = cl.find(',');
        if (c == std::string::npos) continue;
        cache.insert(PairKey{std::stoull(cl.substr(0, c)), std::stoi(cl.substr(c + 1))});
      }
      std::printf("Loaded %zu cached verifications from %s\n", cache.size(), cache_path);
    } else {
      std::printf("No cache yet - will create: %s\n", cache_path);
    }
  }
  std::vector<uint8_t> ok(n, 0);
  std::vector<size_t> todo;
  size_t cached = 0;
  for (size_t i = 0; i < n; ++i) {
    if (cache.count(PairKey{p_after[i], gaps[i]})) {
      ok[i] = 1;
      ++cached;
    } else {
      todo.push_back(i);
    }
  }
  std::printf("Cached: %zu, To verify: %zu\n", cached, todo.size());

  if (!todo.empty()) {
    uint64_t max_p = 0;
    for (size_t i : todo) max_p = p_after[i] > max_p ? p_after[i] : max_p;
    voss_ctx* ctx = nullptr;
    int rc = voss_ctx_create(0, max_p < 8 ? 8 : (max_p > (1ull << 62) ? (1ull << 62) : max_p + 1), &ctx);
    if (rc != VOSS_OK) {
      std::fprintf(stderr, "voss_ctx_create failed: %s\n", voss_last_error());
      return 1;
    }
    std::vector<uint64_t> tp(todo.size());
    std::vector<int32_t> tg(todo.size());
    std::vector<uint8_t> tok(todo.size(), 0);
    for (size_t k = 0; k < todo.size(); ++k) {
      tp[k] = p_after[todo[k]];
      tg[k] = gaps[todo[k]];
    }
    std::printf("Verifying %zu gaps on the GPU...\n", todo.size());
    rc = voss_prove_gaps(ctx, tp.data(), tg.data(), tp.size(), tok.data());
    voss_ctx_destroy(ctx);
    if (rc != VOSS_OK) {
      std::fprintf(stderr, "voss_prove_gaps failed: %s\n", voss_last_error());
      return 1;
    }
    for (size_t k = 0; k < todo.size(); ++k) ok[todo[k]] = tok[k];
  }
  long long verified = 0, failed = 0;
  for (size_t i = 0; i < n; ++i) (ok[i] ? verified : failed)++;

  {
    std::ifstream check(cache_path);
    const bool exists = check.good();
    check.close();
    std::ofstream cf(cache_path, std::ios::app);
    if (!exists) cf << "p_after,gap\n";
    size_t appended = 0;
    for (size_t i : todo)
      if (ok[i]) {
        cf << p_after[i] << "," << gaps[i] << "\n";
        ++appended;
      }
    std::printf("Appended %zu new verifications to cache\n", appended);
  }
  {
    std::ofstream fout(output);
    fout << "position,gap,merit,verified\n";
    char buf[160];
    for (size_t i = 0; i < n; ++i) {
      std::snprintf(buf, sizeof(buf), "%llu,%d,%.6f,%d", (unsigned long long)p_after[i], gaps[i], merits[i],
                    (int)ok[i]);
      fout << buf << "\n";
    }
  }
  const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("\n============================================================\n");
  std::printf("GPU VERIFIER RESULT (cached)\n");
  std::printf("============================================================\n");
  std::printf("Total gaps:    %zu\n", n);
  std::printf("Cached:        %zu  (%.1f%%)\n", cached, 100.0 * cached / n);
  std::printf("Newly verify:  %zu\n", todo.size());
  std::printf("Verified:      %lld\n", verified);
  std::printf("Failed:        %lld\n", failed);
  std::printf("Duration:      %.2f s\n", dt);
  std::printf("Details:       %s\n", output);
  std::printf("Cache:         %s\n", cache_path);
  std::printf("============================================================\n");
  return failed > 0 ? 1 : 0;
}

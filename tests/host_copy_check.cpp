// host_copy_check.cpp — CPU check of libvoss's threaded host copies (parallel_copy and
// parallel_gather in csrc/voss_api.cpp, used by the request server and the staged Miller-Rabin
// and interval paths): random segment lists, empty segments and every part size must give the
// plain concatenation, with nothing written past it.  Built by tests/test_host_copy.py against the
// library's object files; runs without a GPU (no CUDA call is made).
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "voss_host.h"

using namespace voss_host;

int main() {
  std::mt19937_64 g(20261204);
  int bad = 0;
  for (int trial = 0; trial < 60; ++trial) {
    const size_t nseg = 1 + g() % 40;
    std::vector<std::vector<char>> src(nseg);
    std::vector<CopySeg> segs;
    std::vector<char> ref;
    for (auto& v : src) {
      const size_t n = (g() % 4 == 0) ? 0 : (g() % (3u << 20));
      v.resize(n);
      for (auto& c : v) c = (char)g();
      segs.push_back(CopySeg{v.data(), n});
      ref.insert(ref.end(), v.begin(), v.end());
    }
    const size_t part = (trial % 3 == 0) ? 1 : ((trial % 3 == 1) ? (1u << 20) : (64u << 20));
    std::vector<char> dst(ref.size() + 64, 0x55);
    parallel_gather(dst.data(), segs.data(), segs.size(), part);
    if (std::memcmp(dst.data(), ref.data(), ref.size()) != 0) ++bad, std::printf("gather mismatch, trial %d\n", trial);
    for (size_t i = ref.size(); i < dst.size(); ++i)
      if (dst[i] != 0x55) {
        ++bad, std::printf("gather wrote past the end, trial %d\n", trial);
        break;
      }
    std::vector<char> d2(ref.size() + 64, 0x33);
    parallel_copy(d2.data(), ref.data(), ref.size(), part);
    if (std::memcmp(d2.data(), ref.data(), ref.size()) != 0) ++bad, std::printf("copy mismatch, trial %d\n", trial);
    for (size_t i = ref.size(); i < d2.size(); ++i)
      if (d2[i] != 0x33) {
        ++bad, std::printf("copy wrote past the end, trial %d\n", trial);
        break;
      }
  }
  std::printf("bad=%d\n", bad);
  return bad != 0;
}

// Randomized check of the serving engine's range allocator (syn::RangeAlloc in
// syndrome_b200/csrc/serve.cpp: HARQ accumulators, decoded payloads and staged LLRs):
// allocations never overlap or leave the arena, the used count is exact, and once
// everything is released the free ranges have merged back into one.  Prints "ok" or
// the first violation.
#include <cstdio>
#include <random>
#include <utility>
#include <vector>

#include "serve.h"

int main() {
  const long long n = 100000;
  syn::RangeAlloc ra;
  ra.reset(n);
  std::mt19937 rng(1);
  std::vector<std::pair<long long, long long>> live;
  std::vector<char> owner(n, 0);
  long long used = 0;
  for (int it = 0; it < 200000; ++it) {
    if (live.empty() || rng() % 2) {
      const long long len = 1 + rng() % 3000;
      const long long off = ra.alloc(len);
      if (off < 0) continue;
      for (long long i = off; i < off + len; ++i) {
        if (i >= n || owner[i]) {
          std::printf("overlap or out of range at %lld (alloc %lld + %lld)\n", i, off, len);
          return 1;
        }
        owner[i] = 1;
      }
      live.push_back({off, len});
      used += len;
    } else {
      const size_t k = rng() % live.size();
      ra.release(live[k].first);
      for (long long i = live[k].first; i < live[k].first + live[k].second; ++i) owner[i] = 0;
      used -= live[k].second;
      live[k] = live.back();
      live.pop_back();
    }
    if (ra.used != used) {
      std::printf("used %lld, expected %lld after step %d\n", ra.used, used, it);
      return 1;
    }
  }
  for (const auto& l : live) ra.release(l.first);
  if (ra.used != 0 || ra.alloc(n) != 0) {
    std::printf("free ranges did not merge back into one\n");
    return 1;
  }
  std::printf("ok\n");
  return 0;
}

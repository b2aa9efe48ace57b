// Test program for bbtc_b200/csrc/hybrid_core.hpp on the CPU: the CPU task
// count and the GPU/CPU claim protocol, with a stand-in for the GPU side that
// counts its ranges with the same CPU counter.
//
// usage:
//   hybrid_harness <graph> <tasks> tasks
//       prints the count of every task, one per line
//   hybrid_harness <graph> <tasks> run <border> <workers> <gpu_us> <gpu_fail_call>
//       runs the protocol; the stand-in GPU sleeps gpu_us per task of each
//       launch and returns BBTC_ERR_CUDA (-2) on launch number gpu_fail_call
//       (0 = never).  Prints "rc out gpu_tasks cpu_tasks gpu_launches sep
//       gpu_count cpu_count", then per task how often it was counted and by
//       which side ("<times> G" or "<times> C").
// graph file: uint32 n, uint32 P, uint64 m, indptr[n+1], indices[m], cuts[P+1]
// tasks file: uint32 ntasks, then ntasks x (ab, bc, ac) uint32
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "hybrid_core.hpp"

using namespace bbtc::hybrid;

template <class T>
static bool rd(FILE* f, T* p, size_t k) {
  return std::fread(p, sizeof(T), k, f) == k;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <graph> <tasks> tasks|run ...\n", argv[0]);
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  uint32_t n = 0, P = 0;
  uint64_t m = 0;
  if (!rd(f, &n, 1) || !rd(f, &P, 1) || !rd(f, &m, 1)) return 2;
  std::vector<uint32_t> indptr(n + 1), indices(m), cuts(P + 1);
  if (!rd(f, indptr.data(), n + 1) || (m && !rd(f, indices.data(), m)) || !rd(f, cuts.data(), P + 1)) return 2;
  std::fclose(f);

  f = std::fopen(argv[2], "rb");
  if (!f) return 2;
  uint32_t nt = 0;
  if (!rd(f, &nt, 1)) return 2;
  std::vector<uint32_t> tk((size_t)nt * 3);
  if (nt && !rd(f, tk.data(), tk.size())) return 2;
  std::fclose(f);

  HostCsr g;
  g.n = n;
  g.m = m;
  g.indptr = indptr.data();
  g.indices = indices.data();
  g.cuts = cuts.data();
  g.P = P;
  if (!check_shape(g)) {
    std::printf("shape\n");
    return 0;
  }
  auto ijk = [&](uint32_t t, uint32_t* i, uint32_t* j, uint32_t* k) {
    *i = tk[3 * (size_t)t] / P;
    *j = tk[3 * (size_t)t] % P;
    *k = tk[3 * (size_t)t + 1] % P;
  };
  const uint32_t width = widest_part(g);

  if (!std::strcmp(argv[3], "tasks")) {
    if (!check_rows(g, 0, n)) {
      std::printf("rows\n");
      return 0;
    }
    TaskCounter tc(width);
    for (uint32_t t = 0; t < nt; t++) {
      uint32_t i, j, k;
      ijk(t, &i, &j, &k);
      std::printf("%llu\n", (unsigned long long)tc.count(g, i, j, k));
    }
    return 0;
  }
  if (std::strcmp(argv[3], "run") || argc < 8) return 2;
  const int32_t border = std::atoi(argv[4]);
  const uint32_t workers = (uint32_t)std::atoi(argv[5]);
  const int gpu_us = std::atoi(argv[6]);
  const int fail_call = std::atoi(argv[7]);

  std::unique_ptr<std::atomic<uint32_t>[]> seen(new std::atomic<uint32_t>[nt ? nt : 1]);
  std::unique_ptr<std::atomic<char>[]> side(new std::atomic<char>[nt ? nt : 1]);
  for (uint32_t t = 0; t < nt; t++) {
    seen[t].store(0);
    side[t].store('-');
  }
  TaskCounter gpu_tc(width);
  std::vector<TaskCounter> cpu_tc(workers, TaskCounter(width));
  int calls = 0;
  auto gpu = [&](uint32_t first, uint32_t last, uint64_t* c) -> int {
    if (++calls == fail_call) return -2;
    *c = 0;
    for (uint32_t t = first; t < last; t++) {
      uint32_t i, j, k;
      ijk(t, &i, &j, &k);
      *c += gpu_tc.count(g, i, j, k);
      seen[t].fetch_add(1);
      side[t].store('G');
      if (gpu_us) std::this_thread::sleep_for(std::chrono::microseconds(gpu_us));
    }
    return 0;
  };
  auto cpu = [&](uint32_t w, uint32_t t) -> uint64_t {
    uint32_t i, j, k;
    ijk(t, &i, &j, &k);
    seen[t].fetch_add(1);
    side[t].store('C');
    return cpu_tc[w].count(g, i, j, k);
  };
  auto prepare = [&](uint32_t w) -> bool {
    uint32_t lo, hi;
    row_share(g, w, workers, &lo, &hi);
    return check_rows(g, lo, hi);
  };
  Stats s;
  uint64_t out = 0;
  const uint32_t sep = separator(border, nt);
  const int rc = run(nt, sep, workers, gpu, cpu, prepare, -4, -3, &out, &s);
  std::printf("%d %llu %u %u %u %u %llu %llu\n", rc, (unsigned long long)out, s.gpu_tasks, s.cpu_tasks,
              s.gpu_launches, sep, (unsigned long long)s.gpu_count, (unsigned long long)s.cpu_count);
  for (uint32_t t = 0; t < nt; t++) std::printf("%u %c\n", seen[t].load(), side[t].load());
  return 0;
}

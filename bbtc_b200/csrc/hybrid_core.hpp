// hybrid_core.hpp -- CPU side of the hybrid GPU + CPU count (no CUDA).
//
// The reference runs one task list on GPU workers and CPU workers at once
// (bb_tc.cpp:142-252): tasks [0, Separator) belong to the GPU; every task at
// or past the Separator is shared.  GPU workers take shared tasks from the
// head in list order and stop at the first one a CPU worker already holds
// (:163-180); CPU workers take tasks from the tail, one at a time, through a
// decrementing counter and a per-task claim flag (:184-197).  The list is
// sorted heaviest first (tasks.hpp:25-28), so the CPU gets the light tail.
//
// Here the same claim protocol runs with one GPU worker (the calling thread,
// which launches the library's persistent count on contiguous ranges of the
// list) and `workers` CPU threads.  The GPU worker claims a range at a time:
// half of the shared tasks the CPU side has not reached yet, at least one, so
// the two sides meet with single-task granularity after about log2(|T|)
// launches.  Every task is claimed exactly once: the tail counter hands each
// position >= Separator to exactly one CPU worker, which either claims it or
// finds it claimed by the GPU; the GPU claims a prefix of the shared region.
//
// TaskCounter is this library's CPU count of one task over the untiled CSR:
// for rows u of part i, for v in N(u) within part j, the ids of N(v) within
// part k are looked up in a stamp array holding N(u) within part k.  This is
// the task sum of TrianglesInADenseTask / TrianglesInASparseTask
// (cpu_dense_kernel.cpp:24-51, cpu_sparse_kernel.cpp:41-59) computed without
// building tiles: a tile row (ab, bc, ac) of the reference is the slice of a
// CSR row between two cuts.
#pragma once

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <memory>
#include <thread>
#include <vector>

namespace bbtc {
namespace hybrid {

// The oriented CSR and its cut vector, as the caller holds them on the host.
// Contract (the upload's): indptr[0] = 0, non-decreasing, indptr[n] = m; rows
// strictly increasing; ids < n; cuts[0] = 0, non-decreasing, cuts[P] >= n.
struct HostCsr {
  uint32_t n = 0;
  uint64_t m = 0;
  const uint32_t* indptr = nullptr;
  const uint32_t* indices = nullptr;
  const uint32_t* cuts = nullptr;
  uint32_t P = 0;
};

// Row pointer and cut checks, O(n + P).  Once they hold, every read the
// counter makes stays inside indptr[0..n] and indices[0..m), whatever the rows
// hold; check_rows then decides whether the count means anything.
inline bool check_shape(const HostCsr& g) {
  if (!g.indptr || !g.cuts || g.P == 0) return false;
  if (g.m > 0 && !g.indices) return false;
  if (g.indptr[0] != 0 || (uint64_t)g.indptr[g.n] != g.m) return false;
  for (uint32_t u = 0; u < g.n; u++)
    if (g.indptr[u + 1] < g.indptr[u]) return false;
  if (g.cuts[0] != 0 || g.cuts[g.P] < g.n) return false;
  for (uint32_t p = 0; p < g.P; p++)
    if (g.cuts[p + 1] < g.cuts[p]) return false;
  return true;
}

// Rows [lo, hi): strictly increasing, every id < n.
inline bool check_rows(const HostCsr& g, uint32_t lo, uint32_t hi) {
  for (uint32_t u = lo; u < hi; u++) {
    const uint32_t* r = g.indices + g.indptr[u];
    const uint32_t d = g.indptr[u + 1] - g.indptr[u];
    for (uint32_t e = 0; e < d; e++) {
      if (r[e] >= g.n) return false;
      if (e > 0 && r[e] <= r[e - 1]) return false;
    }
  }
  return true;
}

// Rows [*lo, *hi) of worker w of W: contiguous, about m / W entries each
// (R-MAT rows are skewed, so equal row counts would not balance the checks).
inline void row_share(const HostCsr& g, uint32_t w, uint32_t W, uint32_t* lo, uint32_t* hi) {
  auto first_row_at = [&](uint32_t part) -> uint32_t {
    if (part == 0) return 0;
    if (part >= W) return g.n;
    const uint64_t e = g.m * part / W;
    return (uint32_t)(std::lower_bound(g.indptr, g.indptr + g.n + 1, e,
                                       [](uint32_t a, uint64_t b) { return (uint64_t)a < b; }) - g.indptr);
  };
  *lo = std::min(first_row_at(w), g.n);
  *hi = std::min(first_row_at(w + 1), g.n);
  if (w + 1 == W) *hi = g.n;
}

// Widest part, clipped to the rows that exist.
inline uint32_t widest_part(const HostCsr& g) {
  uint32_t w = 0;
  for (uint32_t p = 0; p < g.P; p++) {
    const uint32_t lo = std::min(g.cuts[p], g.n), hi = std::min(g.cuts[p + 1], g.n);
    w = std::max(w, hi - lo);
  }
  return w;
}

class TaskCounter {
 public:
  // stamp_words = widest_part(g); allocates (may throw std::bad_alloc).
  explicit TaskCounter(uint32_t stamp_words) : stamp_(std::max<uint32_t>(stamp_words, 1), 0) {}

  // Sum over rows u of part i, v in N(u) within part j, of
  // |N(u) within part k  ∩  N(v) within part k|.
  uint64_t count(const HostCsr& g, uint32_t i, uint32_t j, uint32_t k) {
    const uint32_t ulo = std::min(g.cuts[i], g.n), uhi = std::min(g.cuts[i + 1], g.n);
    const uint32_t jlo = std::min(g.cuts[j], g.n), jhi = std::min(g.cuts[j + 1], g.n);
    const uint32_t klo = std::min(g.cuts[k], g.n), khi = std::min(g.cuts[k + 1], g.n);
    if (ulo >= uhi || jlo >= jhi || klo >= khi) return 0;
    uint64_t total = 0;
    for (uint32_t u = ulo; u < uhi; u++) {
      const uint32_t* rb = g.indices + g.indptr[u];
      const uint32_t* re = g.indices + g.indptr[u + 1];
      const uint32_t* ab = std::lower_bound(rb, re, jlo);
      const uint32_t* ab_end = std::lower_bound(ab, re, jhi);
      if (ab == ab_end) continue;
      const uint32_t* ac = std::lower_bound(rb, re, klo);
      const uint32_t* ac_end = std::lower_bound(ac, re, khi);
      if (ac == ac_end) continue;  // the reference skips rows with an empty ac row
      const uint32_t gen = next_gen();
      for (const uint32_t* w = ac; w < ac_end; w++) stamp_[*w - klo] = gen;
      for (const uint32_t* pv = ab; pv < ab_end; pv++) {
        const uint32_t v = *pv;
        const uint32_t* vb = g.indices + g.indptr[v];
        const uint32_t* ve = g.indices + g.indptr[v + 1];
        const uint32_t* bc = std::lower_bound(vb, ve, klo);
        uint64_t c = 0;
        for (; bc < ve && *bc < khi; bc++) c += stamp_[*bc - klo] == gen;
        total += c;
      }
    }
    return total;
  }

 private:
  uint32_t next_gen() {
    if (++gen_ == 0) {  // wrapped: old stamps could match again
      std::fill(stamp_.begin(), stamp_.end(), 0u);
      gen_ = 1;
    }
    return gen_;
  }
  std::vector<uint32_t> stamp_;
  uint32_t gen_ = 0;
};

struct Stats {
  uint32_t gpu_tasks = 0, cpu_tasks = 0, gpu_launches = 0;
  uint64_t gpu_count = 0, cpu_count = 0;
  double gpu_ms = 0, cpu_ms = 0;  // wall time of the GPU worker / the slowest CPU worker
};

// Separator from --border (bbtc.cu:54-62): -1 or past the end = all tasks on
// the GPU, -2 = half the list, b >= 0 = b.
inline uint32_t separator(int32_t border, uint32_t ntasks) {
  if (border == -1 || (border >= 0 && (uint32_t)border > ntasks)) return ntasks;
  if (border == -2) return ntasks / 2;
  return (uint32_t)border;
}

// Runs the claim protocol over a list of ntasks.
//   gpu(first, last, &count) counts list positions [first, last) on the GPU
//     and returns 0 or a negative status;
//   cpu(worker, t) returns the count of list position t (worker < workers);
//   prepare(worker) runs on each CPU worker before any worker claims a task
//     and returns false to void the count (input checks split over the
//     workers; after a failure no CPU worker counts anything).
// Returns 0, the GPU's failing status, `bad_input` when a prepare failed, or
// `no_threads` when the CPU worker threads could not all be started (then
// nothing was counted).  With workers == 0 the GPU counts the whole list in
// one call.
template <class GpuFn, class CpuFn, class PrepFn>
int run(uint32_t ntasks, uint32_t sep, uint32_t workers, GpuFn gpu, CpuFn cpu, PrepFn prepare, int bad_input,
        int no_threads, uint64_t* out, Stats* st) {
  using clock = std::chrono::steady_clock;
  Stats s;
  *out = 0;
  if (sep > ntasks) sep = ntasks;
  if (ntasks == 0) {
    if (st) *st = s;
    return 0;
  }
  std::unique_ptr<std::atomic<uint8_t>[]> claim(new std::atomic<uint8_t>[ntasks]);
  for (uint32_t t = 0; t < ntasks; t++) claim[t].store(0, std::memory_order_relaxed);
  std::atomic<int64_t> tail{(int64_t)ntasks - 1};
  std::atomic<bool> abort{false}, bad{false};
  std::atomic<uint64_t> cpu_sum{0};
  std::atomic<uint32_t> cpu_tasks{0};
  std::vector<double> cpu_ms(workers, 0.0);

  std::atomic<uint32_t> prepared{0};
  auto cpu_worker = [&](uint32_t w) {
    const auto t0 = clock::now();
    if (!prepare(w)) bad.store(true);
    // No CPU worker counts before every worker's share of the input checks
    // has passed: the counter relies on sorted rows and ids < n.
    prepared.fetch_add(1);
    while (prepared.load() < workers) std::this_thread::yield();
    uint64_t sum = 0;
    uint32_t done = 0;
    int64_t t = bad.load() ? (int64_t)sep - 1 : tail.fetch_sub(1);
    while (t >= (int64_t)sep && !abort.load(std::memory_order_relaxed)) {
      if (!claim[t].exchange(1)) {
        sum += cpu(w, (uint32_t)t);
        done++;
      }
      t = tail.fetch_sub(1);
    }
    cpu_sum.fetch_add(sum);
    cpu_tasks.fetch_add(done);
    cpu_ms[w] = std::chrono::duration<double, std::milli>(clock::now() - t0).count();
  };

  std::vector<std::thread> pool;
  uint32_t started = 0;
  try {
    pool.reserve(workers);
    for (; started < workers; started++) pool.emplace_back(cpu_worker, started);
  } catch (const std::exception&) {
    abort.store(true);                      // started workers claim nothing
    prepared.fetch_add(workers - started);  // and stop waiting for the missing ones
    for (auto& th : pool) th.join();
    if (st) *st = s;
    return no_threads;
  }

  const auto g0 = clock::now();
  int rc = 0;
  if (workers == 0) {
    for (uint32_t t = 0; t < ntasks; t++) claim[t].store(1, std::memory_order_relaxed);
    uint64_t c = 0;
    rc = gpu(0, ntasks, &c);
    s.gpu_count = c;
    s.gpu_tasks = ntasks;
    s.gpu_launches = 1;
  } else {
    // The GPU's own region [0, sep) goes into the first launch together with
    // the first shared range it claims.
    uint32_t first = 0, h = sep;
    bool stop = false;
    while (rc == 0 && !stop && (first < h || h < ntasks)) {
      const int64_t reach = tail.load() + 1;  // positions below this the CPU side has not taken yet
      const uint64_t open = reach > (int64_t)h ? (uint64_t)(reach - h) : 1;
      const uint32_t want = (uint32_t)std::max<uint64_t>(1, open / 2);
      uint32_t q = h;
      while (q < ntasks && q - h < want) {
        if (claim[q].exchange(1)) {  // a CPU worker holds it: the GPU stops here (bb_tc.cpp:163-180)
          stop = true;
          break;
        }
        q++;
      }
      if (q == ntasks) stop = true;
      if (q > first) {
        uint64_t c = 0;
        rc = gpu(first, q, &c);
        s.gpu_count += c;
        s.gpu_tasks += q - first;
        s.gpu_launches++;
      }
      first = h = q;
    }
    if (rc != 0) abort.store(true);
  }
  s.gpu_ms = std::chrono::duration<double, std::milli>(clock::now() - g0).count();
  for (auto& th : pool) th.join();
  s.cpu_count = cpu_sum.load();
  s.cpu_tasks = cpu_tasks.load();
  for (double v : cpu_ms) s.cpu_ms = std::max(s.cpu_ms, v);
  if (st) *st = s;
  if (rc != 0) return rc;
  if (bad.load()) return bad_input;
  *out = s.gpu_count + s.cpu_count;
  return 0;
}

}  // namespace hybrid
}  // namespace bbtc

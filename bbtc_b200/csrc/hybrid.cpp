// hybrid.cpp -- bbtc_count_hybrid: one task list counted by the GPU and by
// CPU worker threads at once, with the reference's border and claim rules
// (bb_tc.cpp:142-252; the protocol and the CPU task count are in
// hybrid_core.hpp).  The GPU side is the library's own count
// (bbtc_count on contiguous ranges of the list); the context's GPU is
// required, and with cpu_workers = 0 every task runs on it.
#include <new>
#include <string>
#include <vector>

#include "hybrid_core.hpp"
#include "internal.h"

using bbtc::fail;

extern "C" int bbtc_count_hybrid(bbtc_ctx* ctx, bbtc_graph* g, const uint32_t* indptr, const uint32_t* indices,
                                 const bbtc_task* tasks, uint32_t ntasks, int32_t border, uint32_t cpu_workers,
                                 const bbtc_opts* opts, uint64_t* out, bbtc_hybrid_stats* stats) {
  bbtc::Range range("bbtc count hybrid");
  if (!ctx || !g || !out) return fail(BBTC_ERR_ARG, "NULL argument");
  if (g->ctx != ctx) return fail(BBTC_ERR_ARG, "graph belongs to another context");
  if (border < -2) return fail(BBTC_ERR_ARG, "border must be -2, -1 or >= 0");
  if (cpu_workers > 1024) return fail(BBTC_ERR_ARG, "cpu_workers must be at most 1024");
  if (cpu_workers > 0 && (!indptr || (g->m > 0 && !indices)))
    return fail(BBTC_ERR_ARG, "CPU workers need the host CSR (indptr, indices)");
  const uint32_t P = g->P;

  std::vector<bbtc_task> list;
  try {
    if (tasks) {
      list.assign(tasks, tasks + ntasks);
    } else {
      // The reference's CUDA driver: TaskList(P), sorted heaviest first (bbtc.cu:36-37).
      uint32_t nt = 0;
      BBTC_TRY(bbtc_task_list(P, nullptr, 0, &nt));
      list.resize(nt);
      BBTC_TRY(bbtc_task_list(P, list.data(), nt, &nt));
      BBTC_TRY(bbtc_sort_tasks(g, list.data(), nt, 1));
    }
  } catch (const std::bad_alloc&) {
    return fail(BBTC_ERR_NOMEM, "host allocation of the task list failed");
  }
  const uint32_t nt = (uint32_t)list.size();
  std::vector<uint32_t> part;  // i, j, k per task
  try {
    part.resize((size_t)nt * 3);
  } catch (const std::bad_alloc&) {
    return fail(BBTC_ERR_NOMEM, "host allocation failed");
  }
  for (uint32_t q = 0; q < nt; q++) {
    const bbtc_task& t = list[q];
    if (t.ab >= P * P || t.bc >= P * P || t.ac >= P * P)
      return fail(BBTC_ERR_ARG, "task " + std::to_string(q) + " names a tile outside the P x P grid");
    const uint32_t i = t.ab / P, j = t.ab % P, k = t.bc % P;
    if (t.bc / P != j || t.ac != i * P + k)
      return fail(BBTC_ERR_ARG, "task " + std::to_string(q) + " is not (ab, bc, ac) = ((i,j), (j,k), (i,k))");
    part[3 * (size_t)q] = i;
    part[3 * (size_t)q + 1] = j;
    part[3 * (size_t)q + 2] = k;
  }

  bbtc::hybrid::HostCsr hc;
  hc.n = g->n;
  hc.m = g->m;
  hc.indptr = indptr;
  hc.indices = indices;
  hc.cuts = g->cuts.data();
  hc.P = P;
  std::vector<bbtc::hybrid::TaskCounter> counters;
  if (cpu_workers > 0) {
    if (!bbtc::hybrid::check_shape(hc))
      return fail(BBTC_ERR_INPUT, "host CSR does not match the graph (indptr[0] = 0, non-decreasing, indptr[n] = m)");
    try {
      counters.reserve(cpu_workers);
      const uint32_t w = bbtc::hybrid::widest_part(hc);
      for (uint32_t i = 0; i < cpu_workers; i++) counters.emplace_back(w);
    } catch (const std::bad_alloc&) {
      return fail(BBTC_ERR_NOMEM, "host allocation of the CPU workers' stamp arrays failed");
    }
  }

  auto gpu = [&](uint32_t first, uint32_t last, uint64_t* c) -> int {
    return bbtc_count(ctx, g, list.data() + first, last - first, -1, opts, c);
  };
  auto cpu = [&](uint32_t w, uint32_t t) -> uint64_t {
    return counters[w].count(hc, part[3 * (size_t)t], part[3 * (size_t)t + 1], part[3 * (size_t)t + 2]);
  };
  auto prepare = [&](uint32_t w) -> bool {
    uint32_t lo, hi;
    bbtc::hybrid::row_share(hc, w, cpu_workers, &lo, &hi);
    return bbtc::hybrid::check_rows(hc, lo, hi);
  };

  bbtc::hybrid::Stats s;
  const uint32_t sep = bbtc::hybrid::separator(border, nt);
  // distinct codes for the protocol's own failures, so that a status the GPU
  // side returned (and its message) passes through unchanged
  constexpr int kBadRows = -1001, kNoThreads = -1002;
  const int rc = bbtc::hybrid::run(nt, sep, cpu_workers, gpu, cpu, prepare, kBadRows, kNoThreads, out, &s);
  if (stats) {
    stats->gpu_tasks = s.gpu_tasks;
    stats->cpu_tasks = s.cpu_tasks;
    stats->gpu_launches = s.gpu_launches;
    stats->separator = sep;
    stats->gpu_count = s.gpu_count;
    stats->cpu_count = s.cpu_count;
    stats->gpu_ms = s.gpu_ms;
    stats->cpu_ms = s.cpu_ms;
  }
  if (rc == kBadRows) return fail(BBTC_ERR_INPUT, "host CSR breaks the input contract (row not strictly increasing or id >= n)");
  if (rc == kNoThreads) return fail(BBTC_ERR_NOMEM, "CPU worker threads could not be started");
  return rc;  // 0, or a failing bbtc_count's status (it has set the message)
}

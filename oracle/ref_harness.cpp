// ref_harness.cpp -- runs the reference's own CPU counting path in-process.
// TEST INFRASTRUCTURE ONLY (parity checker and timed CPU baseline); the
// library never links it.  It is compiled by oracle/Makefile against the
// reference's unmodified headers and sources, found through -I at build time
// (the reference is a single translation unit: include/triangle_counting/
// bb_tc.h includes its .cpp files), and the result goes to oracle/_ref/.
//
// The call sequence is the CPU driver's (src/bbtc.cpp:115-160) without file
// I/O or partitioning: BlockCSR(cuts, x_adj, adj) -> tasks::TaskList ->
// tasks::SortTasks -> BBTc -> InitFlags -> Separator = border 0 (the CPU
// build's default, include/utils/utils.hpp:26 with src/bbtc.cpp:139-147,
// which hands every task to the CPU workers) -> ResetFlags + NoOfTriangles
// per repeat, timed like the "Triangle Counting Execution Time (s)" region.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <vector>

#include "bb_tc.h"
#include "block_csr.h"
#include "definitions.h"
#include "tasks.hpp"
#include "SARMA/include/sarma.hpp"

extern "C" int ref_count(uint32_t n, const uint32_t* indptr, const uint32_t* indices, const uint32_t* cuts,
                         uint32_t P, int nthreads, int repeat, uint64_t* out, double* seconds) {
  if (!indptr || !cuts || !out || P < 1 || repeat < 1) return -1;
  if (nthreads > 0) omp_set_num_threads(nthreads);
  std::vector<Vertex> vcuts(cuts, cuts + P + 1);
  std::vector<Ordinal> x_adj(indptr, indptr + (size_t)n + 1);
  std::vector<Vertex> adj(indices, indices + indptr[n]);
  BlockCSR<Ordinal, Vertex> st(vcuts, x_adj, adj);
  auto t_list = tasks::TaskList(P);
  tasks::SortTasks(t_list, st);
  BBTc bbtc(&st, t_list, P);
  bbtc.InitFlags();
  bbtc.Separator = 0;
  unsigned long long count = 0;
  for (int r = 0; r < repeat; r++) {
    bbtc.ResetFlags();
    const auto t0 = std::chrono::steady_clock::now();
    count = bbtc.NoOfTriangles();
    const auto t1 = std::chrono::steady_clock::now();
    if (seconds) seconds[r] = std::chrono::duration<double>(t1 - t0).count();
  }
  *out = count;
  st.CleanUp();
  bbtc.CleanUp();
  return 0;
}

// The reference's own cut vector for an oriented CSR: the partitioning step
// of utils::ReadGraph (include/utils/utils.hpp:271-288) after the oriented
// graph A_ord is in memory -- the sampled copy A_sp = A_ord.sparsify(
// get_prob(NNZ, p, p, 10.), 1091467301), then uni on A_sp, n1d on A_ord's
// row pointers, rac on A_ord, pal (anything else) on A_sp after get_sps(),
// and cuts[p] = N + 1.  alg: 0 uni, 1 n1d, 2 pal, 3 rac.  Writes P + 1 cuts.
extern "C" int ref_cuts(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P, int alg,
                        uint32_t* cuts_out) {
  if (!indptr || !cuts_out || P < 1) return -1;
  std::vector<Ordinal> ip(indptr, indptr + (size_t)n + 1);
  std::vector<Ordinal> ix(indices, indices + indptr[n]);
  auto A_ord = std::make_shared<sarma::Matrix<Ordinal, Ordinal>>(
      sarma::Matrix<Ordinal, Ordinal>(ip, ix, ix, ip.size()));
  auto A_sp = std::make_shared<sarma::Matrix<Ordinal, Ordinal>>(
      A_ord->sparsify(sarma::utils::get_prob(A_ord->NNZ(), (Ordinal)P, (Ordinal)P, 10.), 1091467301));
  std::vector<Vertex> cuts;
  const Vertex p = (Vertex)P;
  if (alg == 0) {
    cuts = sarma::uniform::partition<Ordinal, Ordinal>(*A_sp, p);
  } else if (alg == 1) {
    cuts = sarma::nicol1d::partition<Ordinal, Ordinal>(A_ord->indptr, p);
  } else if (alg == 3) {
    cuts = sarma::refine_a_cut::partition<Ordinal, Ordinal>(*A_ord, p);
  } else {
    A_sp->get_sps();
    cuts = sarma::probe_a_load::partition<Ordinal, Ordinal>(*A_sp, p);
  }
  if (cuts.size() != (size_t)P + 1) return -2;
  cuts[p] = A_ord->N() + 1;
  for (uint32_t i = 0; i <= P; i++) cuts_out[i] = (uint32_t)cuts[i];
  return 0;
}

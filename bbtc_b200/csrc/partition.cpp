// Symmetric cut vectors for the 2D block CSR: uni, n1d, pal and rac.
//
// The reference takes these from the vendored SARMA library; the call site is
// include/utils/utils.hpp:271-288.  These are independent implementations of
// the same published algorithms.  The triangle count does not depend on the
// cuts, so they need not agree with SARMA cut for cut.
//
//  * uni (SARMA algorithms/uniform.hpp:20-27): cuts[i] = i*N/P.
//  * n1d (Nicol, "Rectilinear partitioning of irregular data parallel
//    computations", JPDC 1994): the P-way contiguous split of the rows that
//    minimises the largest stripe nnz.  Found here by a binary search on the
//    bottleneck with a greedy probe over the row-pointer prefix, which gives
//    the same optimum (the cuts are the greedy ones at that optimum, as
//    SARMA's Nicol search returns).  (The reference passes the row-pointer array itself as
//    the per-row load, utils.hpp:281 with nicol1d.hpp:284-291; here the load
//    of a row is its nnz.)
//  * pal ("probe a load", SARMA algorithms/probe_a_load.hpp:29-89): one cut
//    vector for rows and columns.  A probe for a load bound L grows the cuts
//    greedily, each new cut as far right as possible while every tile fixed by
//    it (the new row stripe and the new column stripe, up to the new cut) has
//    at most L nonzeros; a binary search finds the smallest L whose probe
//    covers all rows.  As in the reference (utils.hpp:271-273,
//    SARMA tools/utils.hpp:20-25), the loads are taken on a uniform sample of
//    the nonzeros with keep probability min(1, (10P)^2 / nnz).
//  * rac ("refine a cut", SARMA algorithms/refine_a_cut.hpp:43-70,
//    :129-186; the reference calls it on the whole matrix, utils.hpp:282-283):
//    starting from the trivial cuts [0, N, ..., N], each refinement weighs a
//    row by its largest nonzero count inside one column part of the current
//    cuts and takes the optimal contiguous split of those weights; the
//    direction (rows of A or of its transpose) is the one whose first
//    refinement gives the smaller largest tile, refined max(10, P) times.
//    Deterministic, so its cuts equal SARMA's (tests/test_oracle.py).
//
// All four return P+1 cuts with cuts[0] = 0 and cuts[P] = N.
#include <cstdint>

#include "partition_core.hpp"

extern "C" {

// kind: 0 = uni, 1 = n1d, 2 = pal, 3 = pal with the bisection probe (the
// same cuts as 2, slower; kept to check the sweep probe against), 4 = rac.
// cuts must hold P+1 entries.  Returns 0, or -1 for bad arguments.
int bbtcp_cuts(int kind, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P,
               uint64_t seed, uint32_t* cuts) {
  if (!cuts || P < 1 || (kind != 0 && (!indptr || (indptr[n] && !indices)))) return -1;
  if (n == 0) {
    for (uint32_t i = 0; i <= P; i++) cuts[i] = 0;
    return 0;
  }
  switch (kind) {
    case 0: uniform_cuts(n, P, cuts); return 0;
    case 1: n1d_cuts(n, indptr, P, cuts); return 0;
    case 2: pal_cuts_fast(n, indptr, indices, P, seed, cuts); return 0;
    case 3: pal_cuts_bisect(n, indptr, indices, P, seed, cuts); return 0;
    case 4: rac_cuts(n, indptr, indices, P, cuts); return 0;
    default: return -1;
  }
}

}  // extern "C"

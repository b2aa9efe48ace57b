// Symmetric cut vectors for the 2D block CSR: uni, n1d and pal.
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
//    the same optimum.  (The reference passes the row-pointer array itself as
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
//
// All three return P+1 cuts with cuts[0] = 0 and cuts[P] = N.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

inline uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

void uniform_cuts(uint32_t n, uint32_t P, uint32_t* cuts) {
  for (uint32_t i = 0; i <= P; i++) cuts[i] = (uint32_t)((uint64_t)i * n / P);
}

// greedy: can rows be split into <= P stripes of nnz <= B?
bool n1d_probe(uint32_t n, const uint32_t* indptr, uint32_t P, uint64_t B, uint32_t* cuts) {
  uint32_t start = 0;
  uint32_t k = 0;
  if (cuts) cuts[0] = 0;
  while (start < n) {
    if (k == P) return false;
    // furthest end with indptr[end] - indptr[start] <= B
    const uint64_t limit = (uint64_t)indptr[start] + B;
    const uint32_t* it = std::upper_bound(indptr + start, indptr + n + 1, limit,
                                          [](uint64_t v, uint32_t e) { return v < e; });
    uint32_t end = (uint32_t)(it - indptr) - 1;  // last index with indptr <= limit
    if (end <= start) end = start + 1;           // a single row heavier than B
    if ((uint64_t)indptr[end] - indptr[start] > B) return false;
    start = end;
    k++;
    if (cuts) cuts[k] = start;
  }
  if (cuts)
    for (uint32_t t = k + 1; t <= P; t++) cuts[t] = n;
  return true;
}

void n1d_cuts(uint32_t n, const uint32_t* indptr, uint32_t P, uint32_t* cuts) {
  uint64_t lo = 0, hi = indptr[n];
  uint64_t maxrow = 0;
  for (uint32_t i = 0; i < n; i++) maxrow = std::max<uint64_t>(maxrow, indptr[i + 1] - indptr[i]);
  lo = std::max<uint64_t>(maxrow, (indptr[n] + P - 1) / P);
  if (lo > hi) hi = lo;
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (n1d_probe(n, indptr, P, mid, nullptr)) hi = mid; else lo = mid + 1;
  }
  n1d_probe(n, indptr, P, lo, cuts);
  // spread any unused stripes as empty parts at the end
  cuts[P] = n;
}

struct Sample {
  std::vector<uint32_t> row_ptr;  // sampled nonzeros bucketed by row (CSR over n)
  std::vector<uint32_t> row_col;
  std::vector<uint32_t> col_ptr;  // the same sample bucketed by column
  std::vector<uint32_t> col_row;
};

// Bernoulli sample of the nonzeros with probability q, seeded.
Sample make_sample(uint32_t n, const uint32_t* indptr, const uint32_t* indices, double q, uint64_t seed) {
  Sample s;
  s.row_ptr.assign((size_t)n + 1, 0);
  std::vector<uint32_t> rows, cols;
  const uint64_t nnz = indptr[n];
  if (q >= 1.0) {
    rows.reserve(nnz);
    cols.reserve(nnz);
    for (uint32_t r = 0; r < n; r++)
      for (uint32_t e = indptr[r]; e < indptr[r + 1]; e++) {
        rows.push_back(r);
        cols.push_back(indices[e]);
      }
  } else {
    // geometric skips between kept nonzeros
    uint64_t state = mix64(seed ^ 0x5A17ull);
    const double lq = std::log1p(-q);
    uint64_t e = 0;
    uint32_t r = 0;
    while (true) {
      state = mix64(state);
      const double u = ((state >> 11) + 0.5) * (1.0 / 9007199254740992.0);
      e += (uint64_t)std::floor(std::log(u) / lq);
      if (e >= nnz) break;
      while (indptr[r + 1] <= e) r++;
      rows.push_back(r);
      cols.push_back(indices[e]);
      e++;
    }
  }
  for (uint32_t r : rows) s.row_ptr[r + 1]++;
  for (uint32_t i = 0; i < n; i++) s.row_ptr[i + 1] += s.row_ptr[i];
  s.row_col.resize(rows.size());
  {
    std::vector<uint32_t> cur(s.row_ptr.begin(), s.row_ptr.end() - 1);
    for (size_t t = 0; t < rows.size(); t++) s.row_col[cur[rows[t]]++] = cols[t];
  }
  s.col_ptr.assign((size_t)n + 1, 0);
  for (uint32_t c : cols) if (c < n) s.col_ptr[c + 1]++;
  for (uint32_t i = 0; i < n; i++) s.col_ptr[i + 1] += s.col_ptr[i];
  s.col_row.resize(s.col_ptr[n]);
  {
    std::vector<uint32_t> cur(s.col_ptr.begin(), s.col_ptr.end() - 1);
    for (size_t t = 0; t < rows.size(); t++)
      if (cols[t] < n) s.col_row[cur[cols[t]]++] = rows[t];
  }
  return s;
}

// Largest load among the tiles fixed when the part [p.back(), m) is added to
// the cut prefix p: the new row stripe against every column stripe up to m,
// and every row stripe up to m against the new column stripe.
uint64_t new_stripe_maxload(const Sample& s, const std::vector<uint32_t>& p, uint32_t m,
                            std::vector<uint64_t>& scratch) {
  const uint32_t lo = p.back();
  const size_t parts = p.size();  // stripes 0..parts-2 exist, parts-1 is the new one
  scratch.assign(parts, 0);
  auto stripe_of = [&](uint32_t x) -> size_t {
    if (x >= lo) return parts - 1;
    return (size_t)(std::upper_bound(p.begin(), p.end(), x) - p.begin()) - 1;
  };
  uint64_t best = 0;
  // row stripe [lo, m) x column stripes (columns < m); the sampled nonzeros of
  // rows [lo, m) are one contiguous run of the row-bucketed sample
  for (uint32_t t = s.row_ptr[lo]; t < s.row_ptr[m]; t++) {
    const uint32_t c = s.row_col[t];
    if (c < m) scratch[stripe_of(c)]++;
  }
  for (auto v : scratch) best = std::max(best, v);
  // row stripes (rows < lo) x column stripe [lo, m); the diagonal tile is above
  scratch.assign(parts, 0);
  for (uint32_t t = s.col_ptr[lo]; t < s.col_ptr[m]; t++) {
    const uint32_t r = s.col_row[t];
    if (r < lo) scratch[stripe_of(r)]++;
  }
  for (auto v : scratch) best = std::max(best, v);
  return best;
}

// Greedy probe for bound L; cuts grow up to P parts (each cut <= UB[t]).
std::vector<uint32_t> pal_probe(const Sample& s, uint32_t n, uint32_t P, uint64_t L,
                                const std::vector<uint32_t>& UB) {
  std::vector<uint32_t> p{0};
  std::vector<uint64_t> scratch;
  while (p.size() < (size_t)P + 1) {
    uint32_t l = p.back(), r = UB[p.size()];
    while (l < r) {
      const uint32_t m = l + 1 + (r - (l + 1)) / 2;
      if (new_stripe_maxload(s, p, m, scratch) <= L) l = m; else r = m - 1;
    }
    if (l == p.back()) {
      while (p.size() < (size_t)P + 1) p.push_back(p.back());
      break;
    }
    p.push_back(l);
  }
  return p;
}

void pal_cuts(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P, uint64_t seed,
              uint32_t* cuts) {
  const uint64_t nnz = indptr[n];
  const double q = std::min(1.0, (10.0 * P) * (10.0 * P) / std::max<double>(1.0, (double)nnz));
  const Sample s = make_sample(n, indptr, indices, q, seed);
  const uint64_t M = s.row_col.size();
  if (M == 0) {
    uniform_cuts(n, P, cuts);
    return;
  }
  uint64_t lo = (M + (uint64_t)P * P - 1) / ((uint64_t)P * P);
  uint64_t hi = M;
  std::vector<uint32_t> UB(P + 1, n);
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    auto p = pal_probe(s, n, P, mid, UB);
    if (p.back() < n) {
      lo = mid + 1;
    } else {
      hi = mid;
      UB = p;
    }
  }
  auto p = pal_probe(s, n, P, hi, UB);
  for (uint32_t i = 0; i <= P; i++) cuts[i] = p[i];
  cuts[0] = 0;
  cuts[P] = n;
}

}  // namespace

extern "C" {

// kind: 0 = uni, 1 = n1d, 2 = pal.  cuts must hold P+1 entries.
// Returns 0, or -1 for bad arguments.
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
    case 2: pal_cuts(n, indptr, indices, P, seed, cuts); return 0;
    default: return -1;
  }
}

}  // extern "C"

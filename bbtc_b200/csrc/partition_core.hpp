// Partitioning algorithms shared by the host library (partition.cpp) and the
// device entry point (partition_dev.cu).  Every function has internal
// linkage in each translation unit that includes this header.
//
// See partition.cpp for what uni, n1d and pal compute and where they come
// from.  pal here has two probe implementations with the same result:
//  * pal_cuts_bisect: for each new cut, a bisection over the rows, each step
//    recounting the tiles the cut fixes (the first implementation);
//  * pal_from_sample: for each new cut, the sampled nonzeros that the cut
//    can fix are read in order of the smallest cut position that includes
//    them (a merge of the row-sorted and the column-sorted sample) until a
//    tile exceeds the bound, so the largest position whose tiles stay within
//    it is found without recounting.  The tile loads only grow with the position,
//    which makes "largest feasible position" well defined and equal for both.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
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

// Greedy probe over a prefix-sum array (n + 1 nondecreasing entries): can
// [0, n) be split into <= P contiguous parts whose sums are <= B?  Each cut is
// the furthest position whose part stays within B; with `cuts`, they are
// written, and unused parts are empty at the end.
template <class T>
bool prefix_probe(uint32_t n, const T* prefix, uint32_t P, uint64_t B, uint32_t* cuts) {
  uint32_t start = 0;
  uint32_t k = 0;
  if (cuts) cuts[0] = 0;
  while (start < n) {
    if (k == P) return false;
    // furthest end with prefix[end] - prefix[start] <= B
    const uint64_t limit = (uint64_t)prefix[start] + B;
    const T* it = std::upper_bound(prefix + start, prefix + n + 1, limit,
                                   [](uint64_t v, T e) { return v < (uint64_t)e; });
    uint32_t end = (uint32_t)(it - prefix) - 1;  // last index with prefix <= limit
    if (end <= start) end = start + 1;           // a single element heavier than B
    if ((uint64_t)prefix[end] - prefix[start] > B) return false;
    start = end;
    k++;
    if (cuts) cuts[k] = start;
  }
  if (cuts)
    for (uint32_t t = k + 1; t <= P; t++) cuts[t] = n;
  return true;
}

// The optimal P-way contiguous split of a prefix-sum array (Nicol, JPDC 1994:
// the smallest largest part): a binary search on the bound with the greedy
// probe, whose cuts at the optimal bound are returned.
template <class T>
void prefix_cuts(uint32_t n, const T* prefix, uint32_t P, uint32_t* cuts) {
  uint64_t maxel = 0;
  for (uint32_t i = 0; i < n; i++) maxel = std::max<uint64_t>(maxel, (uint64_t)prefix[i + 1] - prefix[i]);
  const uint64_t total = (uint64_t)prefix[n] - prefix[0];
  uint64_t lo = std::max<uint64_t>(maxel, (total + P - 1) / P), hi = std::max<uint64_t>(lo, total);
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    if (prefix_probe(n, prefix, P, mid, nullptr)) hi = mid; else lo = mid + 1;
  }
  prefix_probe(n, prefix, P, lo, cuts);
  cuts[P] = n;
}

// greedy: can rows be split into <= P stripes of nnz <= B?
bool n1d_probe(uint32_t n, const uint32_t* indptr, uint32_t P, uint64_t B, uint32_t* cuts) {
  return prefix_probe(n, indptr, P, B, cuts);
}

void n1d_cuts(uint32_t n, const uint32_t* indptr, uint32_t P, uint32_t* cuts) { prefix_cuts(n, indptr, P, cuts); }

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

void pal_cuts_bisect(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P, uint64_t seed,
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


// ---- pal from an explicit sample ------------------------------------------

// Sampled nonzero indices, in increasing order: the same geometric-skip
// stream as make_sample (every index when q >= 1).
std::vector<uint64_t> pal_sample_edges(uint64_t nnz, uint32_t P, uint64_t seed) {
  const double q = std::min(1.0, (10.0 * P) * (10.0 * P) / std::max<double>(1.0, (double)nnz));
  std::vector<uint64_t> out;
  if (q >= 1.0) {
    out.resize(nnz);
    std::iota(out.begin(), out.end(), 0ull);
    return out;
  }
  uint64_t state = mix64(seed ^ 0x5A17ull);
  const double lq = std::log1p(-q);
  uint64_t e = 0;
  while (true) {
    state = mix64(state);
    const double u = ((state >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    e += (uint64_t)std::floor(std::log(u) / lq);
    if (e >= nnz) break;
    out.push_back(e);
    e++;
  }
  return out;
}

struct SortedSample {
  std::vector<uint32_t> row, col;  // by row (the sample is taken in CSR order), then column
  std::vector<uint32_t> crow, ccol;  // the same nonzeros by column, then row
};

// Largest m in [p.back(), R] whose new stripe [p.back(), m) keeps every tile
// it fixes within L (see new_stripe_maxload for the tiles).
//
// A sampled nonzero (r, c) is counted from position m = t on, its threshold:
//  * row stripe tile (r >= lo, column stripe of c): t = max(r, c) + 1;
//  * column stripe tile (r < lo, lo <= c): t = c + 1.
// Those with c <= r come in threshold order along the row-sorted sample;
// the others (c > r, or r < lo) along the column-sorted one.  The two
// streams are merged by threshold and stopped at the first threshold whose
// nonzeros push a tile above L: only the nonzeros below the answer are read.
uint32_t pal_next_cut(const SortedSample& s, const std::vector<uint32_t>& p, uint32_t R, uint64_t L,
                      std::vector<uint64_t>& ca, std::vector<uint64_t>& cb) {
  const uint32_t lo = p.back();
  if (R <= lo) return lo;
  const size_t parts = p.size();
  auto stripe_of = [&](uint32_t x) -> uint32_t {
    if (x >= lo) return (uint32_t)(parts - 1);
    return (uint32_t)(std::upper_bound(p.begin(), p.end(), x) - p.begin()) - 1;
  };
  ca.assign(parts, 0);
  cb.assign(parts, 0);
  // stream 1: row-sorted, rows [lo, R), entries with c <= r (threshold r + 1)
  size_t i = std::lower_bound(s.row.begin(), s.row.end(), lo) - s.row.begin();
  const size_t i_end = std::lower_bound(s.row.begin(), s.row.end(), R) - s.row.begin();
  // stream 2: column-sorted, columns [lo, R), entries with r < lo or lo <= r < c (threshold c + 1)
  size_t j = std::lower_bound(s.ccol.begin(), s.ccol.end(), lo) - s.ccol.begin();
  const size_t j_end = std::lower_bound(s.ccol.begin(), s.ccol.end(), R) - s.ccol.begin();
  auto skip1 = [&] {
    while (i < i_end && s.col[i] > s.row[i]) i++;
  };
  auto skip2 = [&] {
    while (j < j_end && s.crow[j] >= lo && s.crow[j] >= s.ccol[j]) j++;
  };
  skip1();
  skip2();
  while (i < i_end || j < j_end) {
    const uint32_t t1 = i < i_end ? s.row[i] + 1 : 0xffffffffu;
    const uint32_t t2 = j < j_end ? s.ccol[j] + 1 : 0xffffffffu;
    const uint32_t m = std::min(t1, t2);
    bool over = false;
    while (i < i_end && s.row[i] + 1 == m) {
      if (++ca[stripe_of(s.col[i])] > L) over = true;
      i++;
      skip1();
    }
    while (j < j_end && s.ccol[j] + 1 == m) {
      const uint32_t r = s.crow[j];
      uint64_t& c = r < lo ? cb[stripe_of(r)] : ca[parts - 1];  // r < lo: column stripe tile; else diagonal
      if (++c > L) over = true;
      j++;
      skip2();
    }
    if (over) return m - 1;  // m counts a tile above L; every smaller position is within it
  }
  return R;
}

std::vector<uint32_t> pal_probe_sorted(const SortedSample& s, uint32_t P, uint64_t L, const std::vector<uint32_t>& UB) {
  std::vector<uint32_t> p{0};
  std::vector<uint64_t> ca, cb;
  while (p.size() < (size_t)P + 1) {
    const uint32_t l = pal_next_cut(s, p, UB[p.size()], L, ca, cb);
    if (l == p.back()) {
      while (p.size() < (size_t)P + 1) p.push_back(p.back());
      break;
    }
    p.push_back(l);
  }
  return p;
}

// pal cuts from the sampled nonzeros (rows nondecreasing, columns increasing
// within a row: the CSR order of the sample).
void pal_from_sample(uint32_t n, uint32_t P, const std::vector<uint32_t>& rows, const std::vector<uint32_t>& cols,
                     uint32_t* cuts) {
  const uint64_t M = rows.size();
  if (M == 0) {
    uniform_cuts(n, P, cuts);
    return;
  }
  SortedSample s;
  s.row = rows;
  s.col = cols;
  std::vector<uint32_t> idx(M);
  std::iota(idx.begin(), idx.end(), 0u);
  std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    return cols[a] != cols[b] ? cols[a] < cols[b] : rows[a] < rows[b];
  });
  s.crow.resize(M);
  s.ccol.resize(M);
  for (uint64_t t = 0; t < M; t++) {
    s.crow[t] = rows[idx[t]];
    s.ccol[t] = cols[idx[t]];
  }
  uint64_t lo = (M + (uint64_t)P * P - 1) / ((uint64_t)P * P);
  uint64_t hi = M;
  std::vector<uint32_t> UB(P + 1, n);
  while (lo < hi) {
    const uint64_t mid = lo + (hi - lo) / 2;
    auto p = pal_probe_sorted(s, P, mid, UB);
    if (p.back() < n) {
      lo = mid + 1;
    } else {
      hi = mid;
      UB = p;
    }
  }
  auto p = pal_probe_sorted(s, P, hi, UB);
  for (uint32_t i = 0; i <= P; i++) cuts[i] = p[i];
  cuts[0] = 0;
  cuts[P] = n;
}

// pal on a host CSR: sample, look up each sampled nonzero's row, probe.
void pal_cuts_fast(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P, uint64_t seed,
                   uint32_t* cuts) {
  const std::vector<uint64_t> es = pal_sample_edges(indptr[n], P, seed);
  std::vector<uint32_t> rows(es.size()), cols(es.size());
  uint32_t r = 0;
  for (size_t t = 0; t < es.size(); t++) {
    // rows are nondecreasing along the sample: search forward from the last one
    r = (uint32_t)(std::upper_bound(indptr + r, indptr + n + 1, (uint32_t)es[t]) - indptr) - 1;
    rows[t] = r;
    cols[t] = indices[es[t]];
  }
  pal_from_sample(n, P, rows, cols, cuts);
}

// ---- rac: refine a cut ------------------------------------------------------
//
// Symmetric cuts refined one direction at a time (SARMA
// algorithms/refine_a_cut.hpp:43-70, :129-186): given the current cuts, a
// row's weight is its largest count of nonzeros inside one column part; the
// new cuts are the optimal contiguous split of those weights (prefix_cuts).
// The direction is the rows of A or of its transpose, whichever gives the
// smaller largest tile after one refinement from the trivial cuts
// [0, n, ..., n]; that direction is then refined max(10, P) times.

// Row weights under column cuts `cut` (P + 1 entries, nondecreasing, cut[0] =
// 0, every id < cut[P]), summed into prefix (n + 1 entries).
void rac_weights(uint32_t n, const uint32_t* ptr, const uint32_t* idx, const std::vector<uint32_t>& cut,
                 std::vector<uint64_t>& prefix) {
  prefix.assign((size_t)n + 1, 0);
  for (uint32_t i = 0; i < n; i++) {
    uint64_t best = 0, run = 0;
    size_t k = 1;  // the current column part is [cut[k - 1], cut[k])
    for (uint32_t e = ptr[i]; e < ptr[i + 1]; e++) {
      while (idx[e] >= cut[k]) {
        best = std::max(best, run);
        run = 0;
        k++;
      }
      run++;
    }
    prefix[i + 1] = prefix[i] + std::max(best, run);
  }
}

// Largest tile nnz of A under the symmetric cuts.
uint64_t rac_maxload(uint32_t n, const uint32_t* indptr, const uint32_t* indices, const std::vector<uint32_t>& cut) {
  const size_t P = cut.size() - 1;
  std::vector<uint64_t> tile(P * P, 0);
  size_t x = 0;
  for (uint32_t i = 0; i < n; i++) {
    while (i >= cut[x + 1]) x++;
    for (uint32_t e = indptr[i]; e < indptr[i + 1]; e++) {
      const size_t y = (size_t)(std::upper_bound(cut.begin(), cut.end(), indices[e]) - cut.begin()) - 1;
      tile[x * P + y]++;
    }
  }
  return tile.empty() ? 0 : *std::max_element(tile.begin(), tile.end());
}

void rac_cuts(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint32_t P, uint32_t* cuts) {
  // the transpose, rows sorted (a counting sort by column, rows in order)
  const uint64_t m = indptr[n];
  std::vector<uint32_t> tptr((size_t)n + 1, 0), tidx(m);
  for (uint64_t e = 0; e < m; e++) tptr[indices[e] + 1]++;
  for (uint32_t i = 0; i < n; i++) tptr[i + 1] += tptr[i];
  {
    std::vector<uint32_t> fill(tptr.begin(), tptr.end() - 1);
    for (uint32_t i = 0; i < n; i++)
      for (uint32_t e = indptr[i]; e < indptr[i + 1]; e++) tidx[fill[indices[e]]++] = i;
  }
  std::vector<uint64_t> prefix;
  auto refine = [&](bool transposed, const std::vector<uint32_t>& prev) {
    if (transposed) rac_weights(n, tptr.data(), tidx.data(), prev, prefix);
    else rac_weights(n, indptr, indices, prev, prefix);
    std::vector<uint32_t> next(prev.size());
    prefix_cuts(n, prefix.data(), (uint32_t)prev.size() - 1, next.data());
    return next;
  };
  std::vector<uint32_t> start(P + 1, n);
  start[0] = 0;
  const uint64_t load_rows = rac_maxload(n, indptr, indices, refine(false, start));
  const uint64_t load_cols = rac_maxload(n, indptr, indices, refine(true, start));
  const bool transposed = load_cols < load_rows;
  std::vector<uint32_t> cur = start;
  const uint32_t iters = std::max<uint32_t>(10, P);
  for (uint32_t it = 0; it < iters; it++) cur = refine(transposed, cur);
  std::copy(cur.begin(), cur.end(), cuts);
}

}  // namespace

// Seeded synthetic graphs and host-side preprocessing for bbtc_b200.
//
// Produces the input contract of the counting path: an int32 CSR that is
// symmetrised, free of self-loops and duplicate edges, relabelled by
// ascending (degree, id) and oriented from the lower to the higher new id,
// with every row sorted.  This is the graph the reference builds in
// include/utils/utils.hpp:172-258 (A ∪ Aᵀ without the diagonal) followed by
// SARMA's Matrix::order(ASC, triangular=true)
// (include/utils/SARMA/include/data_structures/csr_matrix.hpp:503-584).
// The reference breaks degree ties with an unstable std::sort; here ties go
// by original id, which makes the relabelling a total order.  The triangle
// count does not depend on the tie order.
//
// Generators (all deterministic for a given seed, independent of the thread
// count, because every random draw comes from a counter-based stream keyed by
// (seed, item index)):
//   * R-MAT: `ef << scale` pairs, per-bit quadrant draw with probabilities
//     a, b, c, d = 1-a-b-c (Chakrabarti, Zhan, Faloutsos, SDM 2004).
//   * Chung-Lu: expected-degree model, edge (i, j) kept with probability
//     min(1, w_i w_j / sum(w)), drawn by Miller & Hagberg's skipping method
//     ("Efficient generation of networks with given expected degrees",
//     WAW 2011).  Weights w_i = C (i + i0)^(-1/(gamma-1)); i0 and C are set
//     so that the mean weight is `mean_deg` and the largest is `max_deg`.
//   * Random geometric graph: n uniform points in the unit square, an edge
//     between every pair closer than `radius` (grid bucketing).
#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

namespace {

inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// A small counter-based stream: state seeded from (seed, index), advanced by
// the splitmix64 increment.
struct Stream {
  uint64_t s;
  Stream(uint64_t seed, uint64_t index)
      : s(splitmix64(seed * 0xD1B54A32D192ED03ull ^ splitmix64(index + 0x632BE59BD9B4E019ull))) {}
  inline uint64_t next() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  // uniform in [0, 1) with 53 random bits
  inline double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Csr {
  uint32_t n = 0;
  std::vector<uint32_t> indptr;   // n + 1
  std::vector<uint32_t> indices;  // m
  uint64_t m_raw = 0;             // pairs generated before cleaning
};

// Exclusive scan of counts[0..n) into offsets[0..n]; returns the total.
uint64_t exclusive_scan(const std::vector<uint32_t>& counts, std::vector<uint64_t>& offsets) {
  const size_t n = counts.size();
  offsets.assign(n + 1, 0);
  for (size_t i = 0; i < n; i++) offsets[i + 1] = offsets[i] + counts[i];
  return offsets[n];
}

// Symmetrise, drop self-loops and duplicates, relabel by (degree, id)
// ascending and orient low -> high.  `src`/`dst` hold m raw pairs.
int clean_and_orient(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m, Csr* out) {
  // 1. bucket every non-loop pair under its smaller endpoint
  std::vector<std::atomic<uint32_t>> cnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) cnt[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)m; e++) {
    const uint32_t u = src[e], v = dst[e];
    if (u == v || u >= n || v >= n) continue;
    cnt[std::min(u, v)].fetch_add(1, std::memory_order_relaxed);
  }
  std::vector<uint64_t> off(n + 1, 0);
  for (uint32_t i = 0; i < n; i++) off[i + 1] = off[i] + cnt[i].load(std::memory_order_relaxed);
  std::vector<uint32_t> hi(off[n]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) cnt[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)m; e++) {
    const uint32_t u = src[e], v = dst[e];
    if (u == v || u >= n || v >= n) continue;
    const uint32_t lo = std::min(u, v);
    const uint32_t pos = cnt[lo].fetch_add(1, std::memory_order_relaxed);
    hi[off[lo] + pos] = std::max(u, v);
  }
  // 2. sort + unique per row
  std::vector<uint32_t> ucnt(n, 0);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    uint32_t* b = hi.data() + off[i];
    uint32_t* e = hi.data() + off[i + 1];
    std::sort(b, e);
    ucnt[i] = (uint32_t)(std::unique(b, e) - b);
  }
  // 3. undirected degrees
  std::vector<std::atomic<uint32_t>> deg(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) deg[i].store(ucnt[i], std::memory_order_relaxed);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; i++)
    for (uint32_t k = 0; k < ucnt[i]; k++) deg[hi[off[i] + k]].fetch_add(1, std::memory_order_relaxed);
  // 4. rank by (degree, id) ascending: counting sort by degree, ids in order
  uint32_t maxdeg = 0;
  for (uint32_t i = 0; i < n; i++) maxdeg = std::max(maxdeg, deg[i].load(std::memory_order_relaxed));
  std::vector<uint64_t> dstart((size_t)maxdeg + 2, 0);
  for (uint32_t i = 0; i < n; i++) dstart[deg[i].load(std::memory_order_relaxed) + 1]++;
  for (size_t d = 1; d < dstart.size(); d++) dstart[d] += dstart[d - 1];
  std::vector<uint32_t> rank(n);
  for (uint32_t i = 0; i < n; i++) rank[i] = (uint32_t)(dstart[deg[i].load(std::memory_order_relaxed)]++);
  // 5. oriented CSR in rank ids
  std::vector<std::atomic<uint32_t>> ocnt(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) ocnt[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; i++)
    for (uint32_t k = 0; k < ucnt[i]; k++) {
      const uint32_t a = rank[i], b = rank[hi[off[i] + k]];
      ocnt[std::min(a, b)].fetch_add(1, std::memory_order_relaxed);
    }
  out->n = n;
  out->indptr.assign((size_t)n + 1, 0);
  uint64_t total = 0;
  for (uint32_t i = 0; i < n; i++) {
    out->indptr[i] = (uint32_t)total;
    total += ocnt[i].load(std::memory_order_relaxed);
  }
  if (total >= (1ull << 32)) return -3;  // does not fit the 32-bit CSR
  out->indptr[n] = (uint32_t)total;
  out->indices.assign(total, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) ocnt[i].store(0, std::memory_order_relaxed);
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; i++)
    for (uint32_t k = 0; k < ucnt[i]; k++) {
      const uint32_t a = rank[i], b = rank[hi[off[i] + k]];
      const uint32_t r = std::min(a, b);
      const uint32_t pos = ocnt[r].fetch_add(1, std::memory_order_relaxed);
      out->indices[out->indptr[r] + pos] = std::max(a, b);
    }
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t i = 0; i < (int64_t)n; i++)
    std::sort(out->indices.begin() + out->indptr[i], out->indices.begin() + out->indptr[i + 1]);
  out->m_raw = m;
  return 0;
}

int gen_rmat(int scale, int ef, double a, double b, double c, uint64_t seed, Csr* out) {
  if (scale < 1 || scale > 31 || ef < 1) return -1;
  const uint32_t n = 1u << scale;
  const uint64_t m = (uint64_t)ef << scale;
  std::vector<uint32_t> src(m), dst(m);
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)m; e++) {
    Stream rng(seed, (uint64_t)e);
    uint32_t u = 0, v = 0;
    for (int l = scale - 1; l >= 0; l--) {
      const double r = rng.uniform();
      if (r < a) {
      } else if (r < ab) {
        v |= 1u << l;
      } else if (r < abc) {
        u |= 1u << l;
      } else {
        u |= 1u << l;
        v |= 1u << l;
      }
    }
    src[e] = u;
    dst[e] = v;
  }
  return clean_and_orient(n, src.data(), dst.data(), m, out);
}

// Σ_{i=0}^{n-1} (i + i0)^(-alpha): the first 1024 terms exactly, the tail by
// the midpoint integral (used only to pick i0)
double approx_power_sum(double n, double i0, double alpha) {
  const double head = std::min(n, 1024.0);
  double s = 0;
  for (double i = 0; i < head; i += 1) s += std::pow(i + i0, -alpha);
  if (n > head) {
    const double lo = head + i0 - 0.5, hi = n + i0 - 0.5;
    s += (std::pow(hi, 1.0 - alpha) - std::pow(lo, 1.0 - alpha)) / (1.0 - alpha);
  }
  return s;
}

int gen_chung_lu(uint32_t n, double gamma, double mean_deg, double max_deg, uint64_t seed, Csr* out) {
  if (n < 2 || gamma <= 2.0 || mean_deg <= 0 || max_deg < mean_deg) return -1;
  const double alpha = 1.0 / (gamma - 1.0);
  // pick i0 so that max/mean = n * i0^-alpha / Σ (i+i0)^-alpha
  const double target = max_deg / mean_deg;
  double lo = 1e-3, hi = (double)n;
  for (int it = 0; it < 100; it++) {
    const double mid = std::sqrt(lo * hi);
    const double ratio = n * std::pow(mid, -alpha) / approx_power_sum(n, mid, alpha);
    if (ratio > target) lo = mid; else hi = mid;  // ratio falls as i0 grows
  }
  const double i0 = std::sqrt(lo * hi);
  std::vector<double> w(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) w[i] = std::pow((double)i + i0, -alpha);
  // the sums run in index order: the graph must not depend on the thread count
  double sum = 0;
  for (uint32_t i = 0; i < n; i++) sum += w[i];
  const double scale = mean_deg * n / sum;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) w[i] = std::min(w[i] * scale, max_deg);
  double S = 0;
  for (uint32_t i = 0; i < n; i++) S += w[i];
  // weights are non-increasing in i, as the skipping method requires
  const int nt = omp_get_max_threads();
  std::vector<std::vector<uint32_t>> es(nt), ed(nt);
#pragma omp parallel
  {
    const int t = omp_get_thread_num();
    auto& s_out = es[t];
    auto& d_out = ed[t];
#pragma omp for schedule(dynamic, 256)
    for (int64_t u = 0; u < (int64_t)n - 1; u++) {
      Stream rng(seed, (uint64_t)u);
      uint64_t v = (uint64_t)u + 1;
      double p = std::min(w[u] * w[v] / S, 1.0);
      while (v < n && p > 0) {
        if (p != 1.0) {
          const double r = rng.uniform();
          v += (uint64_t)std::floor(std::log(1.0 - r) / std::log(1.0 - p));
        }
        if (v < n) {
          const double q = std::min(w[u] * w[v] / S, 1.0);
          const double r = rng.uniform();
          if (r < q / p) {
            s_out.push_back((uint32_t)u);
            d_out.push_back((uint32_t)v);
          }
          p = q;
          v += 1;
        }
      }
    }
  }
  size_t m = 0;
  for (auto& v : es) m += v.size();
  std::vector<uint32_t> src(m), dst(m);
  size_t pos = 0;
  for (int t = 0; t < nt; t++) {
    std::copy(es[t].begin(), es[t].end(), src.begin() + pos);
    std::copy(ed[t].begin(), ed[t].end(), dst.begin() + pos);
    pos += es[t].size();
  }
  return clean_and_orient(n, src.data(), dst.data(), m, out);
}

int gen_rgg(uint32_t n, double radius, uint64_t seed, Csr* out) {
  if (n < 2 || radius <= 0 || radius >= 1) return -1;
  std::vector<double> x(n), y(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; i++) {
    Stream rng(seed, (uint64_t)i);
    x[i] = rng.uniform();
    y[i] = rng.uniform();
  }
  const uint32_t G = std::max<uint32_t>(1, (uint32_t)std::floor(1.0 / radius));
  auto cell_of = [&](uint32_t i) {
    const uint32_t cx = std::min<uint32_t>(G - 1, (uint32_t)(x[i] * G));
    const uint32_t cy = std::min<uint32_t>(G - 1, (uint32_t)(y[i] * G));
    return (uint64_t)cy * G + cx;
  };
  std::vector<uint32_t> ccount((size_t)G * G, 0);
  for (uint32_t i = 0; i < n; i++) ccount[cell_of(i)]++;
  std::vector<uint64_t> cstart;
  exclusive_scan(ccount, cstart);
  std::vector<uint32_t> order(n);
  {
    std::vector<uint64_t> cur(cstart.begin(), cstart.end() - 1);
    for (uint32_t i = 0; i < n; i++) order[cur[cell_of(i)]++] = i;
  }
  const double r2 = radius * radius;
  const int nt = omp_get_max_threads();
  std::vector<std::vector<uint32_t>> es(nt), ed(nt);
#pragma omp parallel
  {
    const int t = omp_get_thread_num();
#pragma omp for schedule(dynamic, 64)
    for (int64_t cyx = 0; cyx < (int64_t)G * G; cyx++) {
      const int64_t cy = cyx / G, cx = cyx % G;
      for (uint64_t a = cstart[cyx]; a < cstart[cyx + 1]; a++) {
        const uint32_t i = order[a];
        for (int64_t dy = -1; dy <= 1; dy++)
          for (int64_t dx = -1; dx <= 1; dx++) {
            const int64_t ny = cy + dy, nx = cx + dx;
            if (ny < 0 || nx < 0 || ny >= (int64_t)G || nx >= (int64_t)G) continue;
            const uint64_t c2 = (uint64_t)ny * G + nx;
            for (uint64_t b2 = cstart[c2]; b2 < cstart[c2 + 1]; b2++) {
              const uint32_t j = order[b2];
              if (j <= i) continue;
              const double ddx = x[i] - x[j], ddy = y[i] - y[j];
              if (ddx * ddx + ddy * ddy < r2) {
                es[t].push_back(i);
                ed[t].push_back(j);
              }
            }
          }
      }
    }
  }
  size_t m = 0;
  for (auto& v : es) m += v.size();
  std::vector<uint32_t> src(m), dst(m);
  size_t pos = 0;
  for (int t = 0; t < nt; t++) {
    std::copy(es[t].begin(), es[t].end(), src.begin() + pos);
    std::copy(ed[t].begin(), ed[t].end(), dst.begin() + pos);
    pos += es[t].size();
  }
  return clean_and_orient(n, src.data(), dst.data(), m, out);
}

template <class F>
int make(void** handle, F&& f) {
  if (!handle) return -1;
  *handle = nullptr;
  Csr* g = new (std::nothrow) Csr();
  if (!g) return -2;
  int rc;
  try {
    rc = f(g);
  } catch (const std::bad_alloc&) {
    rc = -2;
  }
  if (rc != 0) {
    delete g;
    return rc;
  }
  *handle = g;
  return 0;
}

}  // namespace

extern "C" {

// All functions return 0 on success, -1 for bad arguments, -2 when memory
// runs out, -3 when the cleaned graph has 2^32 or more edges.

int bbtcg_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, void** handle) {
  return make(handle, [&](Csr* g) { return gen_rmat(scale, edge_factor, a, b, c, seed, g); });
}

int bbtcg_chung_lu(uint32_t n, double gamma, double mean_deg, double max_deg, uint64_t seed, void** handle) {
  return make(handle, [&](Csr* g) { return gen_chung_lu(n, gamma, mean_deg, max_deg, seed, g); });
}

int bbtcg_rgg(uint32_t n, double radius, uint64_t seed, void** handle) {
  return make(handle, [&](Csr* g) { return gen_rgg(n, radius, seed, g); });
}

// Clean and orient a caller-supplied list of m directed pairs over ids < n.
int bbtcg_from_pairs(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m, void** handle) {
  if (m && (!src || !dst)) return -1;
  return make(handle, [&](Csr* g) { return clean_and_orient(n, src, dst, m, g); });
}

// Wrap an already oriented CSR (copied, not cleaned: the counting library
// checks the input contract on upload).
int bbtcg_from_csr(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m, void** handle) {
  if (!indptr || (m && !indices)) return -1;
  if (m >= (1ull << 32)) return -3;
  return make(handle, [&](Csr* g) {
    g->n = n;
    g->indptr.assign(indptr, indptr + (size_t)n + 1);
    g->indices.assign(indices, indices + m);
    g->m_raw = m;
    return 0;
  });
}

int bbtcg_info(void* handle, uint32_t* n, uint64_t* m, uint64_t* m_raw) {
  if (!handle) return -1;
  const Csr* g = static_cast<const Csr*>(handle);
  if (n) *n = g->n;
  if (m) *m = g->indices.size();
  if (m_raw) *m_raw = g->m_raw;
  return 0;
}

int bbtcg_copy(void* handle, uint32_t* indptr, uint32_t* indices) {
  if (!handle) return -1;
  const Csr* g = static_cast<const Csr*>(handle);
  if (indptr) std::memcpy(indptr, g->indptr.data(), g->indptr.size() * sizeof(uint32_t));
  if (indices && !g->indices.empty())
    std::memcpy(indices, g->indices.data(), g->indices.size() * sizeof(uint32_t));
  return 0;
}

int bbtcg_free(void* handle) {
  delete static_cast<Csr*>(handle);
  return 0;
}

}  // extern "C"

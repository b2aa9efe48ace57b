/* graphs_oracle.c -- seeded synthetic graphs for the reference arm and the
 * parity tests.  TEST INFRASTRUCTURE ONLY: the library never links it.
 *
 * It restates the library's generators (bbtc_b200/csrc/graphgen.cpp) so that
 * the timed reference CPU path can be fed the benchmark graphs without
 * loading any of the library's code, and so that the generators themselves
 * are checked by a second implementation (tests/test_oracle.py compares the
 * two bit for bit):
 *   - the draws: a counter-based stream per item, state
 *     splitmix64(seed * 0xD1B54A32D192ED03 ^ splitmix64(index + 0x632BE59BD9B4E019)),
 *     advanced by the splitmix64 increment; uniforms carry 53 bits;
 *   - R-MAT (Chakrabarti, Zhan, Faloutsos, SDM 2004): per pair, scale
 *     quadrant draws from the top bit down with probabilities a, b, c, d;
 *   - Chung-Lu by Miller & Hagberg's skipping method (WAW 2011), weights
 *     w_i = C (i + i0)^(-1/(gamma-1)) scaled to the mean and capped;
 *   - cleaning as the reference's graph preparation does
 *     (include/utils/utils.hpp:172-258: A ∪ Aᵀ without the diagonal) and its
 *     ascending-degree orientation (SARMA csr_matrix.hpp:503-584), with ties
 *     by id.  The method differs from the library's on purpose: every pair
 *     becomes one 64-bit key (low id, high id), all keys are radix-sorted
 *     and deduplicated at once, and the oriented edges are sorted the same
 *     way, where the library buckets pairs per row and sorts each row.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

typedef struct {
  uint64_t s;
} stream_t;

static stream_t stream_at(uint64_t seed, uint64_t index) {
  stream_t r;
  r.s = splitmix64((seed * 0xD1B54A32D192ED03ull) ^ splitmix64(index + 0x632BE59BD9B4E019ull));
  return r;
}

static uint64_t stream_next(stream_t* r) {
  r->s += 0x9E3779B97F4A7C15ull;
  uint64_t z = r->s;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static double stream_uniform(stream_t* r) { return (double)(stream_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* LSD radix sort of 64-bit keys, 16 bits a pass. */
static int radix_sort_u64(uint64_t* a, uint64_t n) {
  uint64_t* b = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
  uint64_t* cnt = (uint64_t*)malloc(65536 * sizeof(uint64_t));
  if (!b || !cnt) {
    free(b);
    free(cnt);
    return -2;
  }
  uint64_t *src = a, *dst = b;
  for (int shift = 0; shift < 64; shift += 16) {
    memset(cnt, 0, 65536 * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++) cnt[(src[i] >> shift) & 0xffff]++;
    uint64_t sum = 0;
    for (int d = 0; d < 65536; d++) {
      const uint64_t c = cnt[d];
      cnt[d] = sum;
      sum += c;
    }
    for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> shift) & 0xffff]++] = src[i];
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  /* four passes: the sorted keys are back in a */
  free(b);
  free(cnt);
  return 0;
}

/* Keys (low << 32 | high) of m raw pairs -> oriented CSR.  Frees keys. */
static int orient_keys(uint32_t n, uint64_t* keys, uint64_t m, uint32_t** indptr_out, uint32_t** indices_out,
                       uint64_t* m_out) {
  int rc = radix_sort_u64(keys, m);
  if (rc) {
    free(keys);
    return rc;
  }
  uint64_t k = 0;
  for (uint64_t i = 0; i < m; i++)
    if (i == 0 || keys[i] != keys[i - 1]) keys[k++] = keys[i];
  const uint64_t e = k; /* undirected edges, low < high, distinct */
  uint32_t* deg = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
  uint32_t* rank = (uint32_t*)malloc(((size_t)n + 1) * sizeof(uint32_t));
  if (!deg || !rank) {
    free(deg);
    free(rank);
    free(keys);
    return -2;
  }
  uint32_t maxdeg = 0;
  for (uint64_t i = 0; i < e; i++) {
    deg[keys[i] >> 32]++;
    deg[(uint32_t)keys[i]]++;
  }
  for (uint32_t i = 0; i < n; i++)
    if (deg[i] > maxdeg) maxdeg = deg[i];
  /* rank by (degree, id) ascending: ids in order within each degree */
  uint64_t* start = (uint64_t*)calloc((size_t)maxdeg + 2, sizeof(uint64_t));
  if (!start) {
    free(deg);
    free(rank);
    free(keys);
    return -2;
  }
  for (uint32_t i = 0; i < n; i++) start[deg[i] + 1]++;
  for (uint32_t d = 1; d <= maxdeg + 1; d++) start[d] += start[d - 1];
  for (uint32_t i = 0; i < n; i++) rank[i] = (uint32_t)start[deg[i]]++;
  free(start);
  free(deg);
  for (uint64_t i = 0; i < e; i++) {
    const uint32_t a = rank[keys[i] >> 32], b = rank[(uint32_t)keys[i]];
    keys[i] = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
  }
  free(rank);
  rc = radix_sort_u64(keys, e);
  if (rc) {
    free(keys);
    return rc;
  }
  if (e >= (1ull << 32)) {
    free(keys);
    return -3;
  }
  uint32_t* indptr = (uint32_t*)calloc((size_t)n + 1, sizeof(uint32_t));
  uint32_t* indices = (uint32_t*)malloc((e ? e : 1) * sizeof(uint32_t));
  if (!indptr || !indices) {
    free(indptr);
    free(indices);
    free(keys);
    return -2;
  }
  for (uint64_t i = 0; i < e; i++) {
    indptr[(keys[i] >> 32) + 1]++;
    indices[i] = (uint32_t)keys[i];
  }
  for (uint32_t i = 0; i < n; i++) indptr[i + 1] += indptr[i];
  free(keys);
  *indptr_out = indptr;
  *indices_out = indices;
  *m_out = e;
  return 0;
}

/* Key of a raw pair, or ~0 for a self loop / an id >= n. */
static uint64_t pair_key(uint32_t n, uint32_t u, uint32_t v) {
  if (u == v || u >= n || v >= n) return ~0ull;
  return u < v ? ((uint64_t)u << 32 | v) : ((uint64_t)v << 32 | u);
}

/* Drops the ~0 keys (skipped pairs) in place; returns the count kept. */
static uint64_t compact(uint64_t* keys, uint64_t m) {
  uint64_t k = 0;
  for (uint64_t i = 0; i < m; i++)
    if (keys[i] != ~0ull) keys[k++] = keys[i];
  return k;
}

int oracle_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed, uint32_t* n_out,
                uint64_t* m_out, uint32_t** indptr, uint32_t** indices) {
  if (scale < 1 || scale > 31 || edge_factor < 1 || !n_out || !m_out || !indptr || !indices) return -1;
  const uint32_t n = 1u << scale;
  const uint64_t m = (uint64_t)edge_factor << scale;
  uint64_t* keys = (uint64_t*)malloc(m * sizeof(uint64_t));
  if (!keys) return -2;
  const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < (int64_t)m; e++) {
    stream_t r = stream_at(seed, (uint64_t)e);
    uint32_t u = 0, v = 0;
    for (int l = scale - 1; l >= 0; l--) {
      const double x = stream_uniform(&r);
      if (x < a) {
      } else if (x < ab) {
        v |= 1u << l;
      } else if (x < abc) {
        u |= 1u << l;
      } else {
        u |= 1u << l;
        v |= 1u << l;
      }
    }
    keys[e] = pair_key(n, u, v);
  }
  *n_out = n;
  return orient_keys(n, keys, compact(keys, m), indptr, indices, m_out);
}

/* sum_{i<n} (i + i0)^-alpha: the first 1024 terms exactly, the tail by the
 * midpoint integral (only used to pick i0) */
static double power_sum(double n, double i0, double alpha) {
  const double head = n < 1024.0 ? n : 1024.0;
  double s = 0;
  for (double i = 0; i < head; i += 1) s += pow(i + i0, -alpha);
  if (n > head) {
    const double lo = head + i0 - 0.5, hi = n + i0 - 0.5;
    s += (pow(hi, 1.0 - alpha) - pow(lo, 1.0 - alpha)) / (1.0 - alpha);
  }
  return s;
}

int oracle_chung_lu(uint32_t n, double gamma, double mean_deg, double max_deg, uint64_t seed, uint64_t* m_out,
                    uint32_t** indptr, uint32_t** indices) {
  if (n < 2 || gamma <= 2.0 || mean_deg <= 0 || max_deg < mean_deg || !m_out || !indptr || !indices) return -1;
  const double alpha = 1.0 / (gamma - 1.0);
  /* i0: max / mean = n i0^-alpha / sum (i + i0)^-alpha, by bisection in log space */
  const double target = max_deg / mean_deg;
  double lo = 1e-3, hi = (double)n;
  for (int it = 0; it < 100; it++) {
    const double mid = sqrt(lo * hi);
    const double ratio = n * pow(mid, -alpha) / power_sum(n, mid, alpha);
    if (ratio > target) lo = mid; else hi = mid;
  }
  const double i0 = sqrt(lo * hi);
  double* w = (double*)malloc((size_t)n * sizeof(double));
  if (!w) return -2;
  double sum = 0, S = 0;
  for (uint32_t i = 0; i < n; i++) {
    w[i] = pow((double)i + i0, -alpha);
    sum += w[i];
  }
  const double scale = mean_deg * n / sum;
  for (uint32_t i = 0; i < n; i++) {
    const double x = w[i] * scale;
    w[i] = max_deg < x ? max_deg : x;
    S += w[i];
  }
  /* pairs (u, v > u): skip to the next candidate v by a geometric jump at the
   * current probability p, accept it with probability q / p */
  uint64_t cap = (uint64_t)(mean_deg * n) + 1024, m = 0;
  uint64_t* keys = (uint64_t*)malloc(cap * sizeof(uint64_t));
  if (!keys) {
    free(w);
    return -2;
  }
  for (uint32_t u = 0; u + 1 < n; u++) {
    stream_t r = stream_at(seed, u);
    uint64_t v = (uint64_t)u + 1;
    double p = w[u] * w[v] / S;
    if (p > 1.0) p = 1.0;
    while (v < n && p > 0) {
      if (p != 1.0) v += (uint64_t)floor(log(1.0 - stream_uniform(&r)) / log(1.0 - p));
      if (v < n) {
        double q = w[u] * w[v] / S;
        if (q > 1.0) q = 1.0;
        if (stream_uniform(&r) < q / p) {
          if (m == cap) {
            cap *= 2;
            uint64_t* k2 = (uint64_t*)realloc(keys, cap * sizeof(uint64_t));
            if (!k2) {
              free(keys);
              free(w);
              return -2;
            }
            keys = k2;
          }
          keys[m++] = pair_key(n, u, (uint32_t)v);
        }
        p = q;
        v += 1;
      }
    }
  }
  free(w);
  return orient_keys(n, keys, compact(keys, m), indptr, indices, m_out);
}

void oracle_free(void* p) { free(p); }

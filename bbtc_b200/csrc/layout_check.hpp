// Host-side check of a block-CSR layout read back from the device.
//
// The reference builds its tiles on the host and never checks them
// (src/data_structures/block_csr.cpp:288-376); here the layout is built by
// device kernels, and this checker states what every kernel that reads it
// relies on, over plain host arrays (no CUDA types, so it also compiles into
// host-only test programs):
//
//   * the oriented CSR: indptr[0] = 0, non-decreasing, indptr[n] = m; rows
//     strictly increasing; ids < n;
//   * the word-compressed rows: wptr[0] = 0, non-decreasing; within a row the
//     32-id words strictly increase, masks are non-zero, and the pairs expand
//     to exactly the row's ids;
//   * the pivot descriptors: per vertex its row start, pair start, first and
//     last id;
//   * each block CSR (forward: rows of part x, columns of part y; reversed:
//     the same with the transposed graph): row-pointer segments start on
//     16-byte boundaries, stay inside the pool and do not overlap; a tile's
//     segment starts at 0, never decreases and ends at the tile's nnz; column
//     segments of non-empty tiles are 16-byte aligned, disjoint and inside the
//     pool (empty tiles have none); every tile row is strictly increasing with
//     columns < the tile's width, and equals the source row's ids inside the
//     column part (so every edge sits in exactly one tile); the tile's longest
//     row and non-empty row count are right; the row index of every 32nd entry
//     names the row holding that entry;
//   * the reversed tiles' records: entry (v, u) of row part x holds the end of
//     row u's pairs and its first pair: the one that contains v, or -- when
//     the first id L of v's row at or above cuts[x] lies in a lower 32-id
//     word than v -- the first pair of row u whose word is >= L / 32.
// Each check returns "" or a message naming the first broken rule.
#pragma once

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

namespace bbtc {
namespace check {

constexpr uint64_t kNoSeg = ~0ull;  // column offset of an empty tile

struct Csr {
  uint32_t n = 0;
  uint64_t m = 0;
  const uint32_t* indptr = nullptr;  // n + 1
  const uint32_t* indices = nullptr;  // m
};

struct Words {
  const uint32_t* wptr = nullptr;   // n + 1 pair offsets
  const uint32_t* pairs = nullptr;  // 2 words a pair: (32-id word index, bit mask)
  uint64_t cap = 0;                 // pairs the buffer holds
};

struct Tiles {
  uint32_t P = 0;
  const uint32_t* cuts = nullptr;   // P + 1
  const uint64_t* rp_off = nullptr; // P * P
  const uint64_t* col_off = nullptr;
  const uint32_t* nnz = nullptr;
  const uint32_t* maxdeg = nullptr;
  const uint32_t* nerows = nullptr;
  const uint32_t* rp = nullptr;
  uint64_t rp_len = 0;
  const uint32_t* col = nullptr;
  uint64_t col_len = 0;
  const uint32_t* erow = nullptr;
  uint64_t erow_len = 0;
  const uint32_t* rec = nullptr;    // reversed tiles: 2 words per column slot, else null
};

inline std::string at(const char* what, uint64_t a, uint64_t b = ~0ull) {
  std::string s = what;
  s += " (";
  s += std::to_string(a);
  if (b != ~0ull) s += ", " + std::to_string(b);
  return s + ")";
}

inline std::string csr(const Csr& g) {
  if (g.indptr[0] != 0) return "indptr[0] != 0";
  if ((uint64_t)g.indptr[g.n] != g.m) return "indptr[n] != m";
  for (uint32_t u = 0; u < g.n; u++) {
    const uint32_t a = g.indptr[u], b = g.indptr[u + 1];
    if (b < a) return at("indptr decreases at row", u);
    for (uint32_t e = a; e < b; e++) {
      if (g.indices[e] >= g.n) return at("id >= n in row", u);
      if (e > a && g.indices[e - 1] >= g.indices[e]) return at("row not strictly increasing", u);
    }
  }
  return "";
}

inline std::string words(const Csr& g, const Words& w) {
  if (w.wptr[0] != 0) return "wptr[0] != 0";
  if (w.wptr[g.n] > w.cap) return "wptr[n] beyond the pair buffer";
  for (uint32_t u = 0; u < g.n; u++) {
    const uint32_t a = w.wptr[u], b = w.wptr[u + 1];
    if (b < a) return at("wptr decreases at row", u);
    uint32_t e = g.indptr[u];
    const uint32_t end = g.indptr[u + 1];
    for (uint32_t p = a; p < b; p++) {
      if (w.pairs[2 * p + 1] == 0) return at("empty mask in row", u, p);
      if (p > a && w.pairs[2 * (p - 1)] >= w.pairs[2 * p]) return at("words not increasing in row", u, p);
    }
    for (uint32_t p = a; p < b; p++) {
      const uint32_t word = w.pairs[2 * p], mask = w.pairs[2 * p + 1];
      for (uint32_t bit = 0; bit < 32; bit++) {
        if (!(mask >> bit & 1)) continue;
        if (e >= end || g.indices[e] != word * 32 + bit) return at("pairs do not expand to row", u, p);
        e++;
      }
    }
    if (e != end) return at("pairs miss ids of row", u);
  }
  return "";
}

// Pivot descriptors (4 words per vertex u <= n): row start, pair start,
// first id and last id of row u (0, 0 for an empty row and for u = n).
inline std::string descs(const Csr& g, const Words& w, const uint32_t* desc) {
  for (uint32_t u = 0; u <= g.n; u++) {
    const uint32_t* d = desc + 4 * (uint64_t)u;
    const bool has = u < g.n && g.indptr[u + 1] > g.indptr[u];
    const uint32_t first = has ? g.indices[g.indptr[u]] : 0, last = has ? g.indices[g.indptr[u + 1] - 1] : 0;
    if (d[0] != g.indptr[u] || d[1] != w.wptr[u] || d[2] != first || d[3] != last)
      return at("pivot descriptor differs from the row, vertex", u);
  }
  return "";
}

// Transposed CSR of g (columns ascending within each row).
inline void transpose(const Csr& g, std::vector<uint32_t>& tp, std::vector<uint32_t>& tc) {
  tp.assign((size_t)g.n + 1, 0);
  tc.assign((size_t)g.m, 0);
  for (uint64_t e = 0; e < g.m; e++) tp[g.indices[e] + 1]++;
  for (uint32_t v = 0; v < g.n; v++) tp[v + 1] += tp[v];
  std::vector<uint32_t> cur(tp.begin(), tp.end() - 1);
  for (uint32_t u = 0; u < g.n; u++)
    for (uint32_t e = g.indptr[u]; e < g.indptr[u + 1]; e++) tc[cur[g.indices[e]]++] = u;
}

// Segments [off, off + len) (len > 0) must be pairwise disjoint.
inline bool disjoint(std::vector<std::pair<uint64_t, uint64_t>> seg) {
  std::sort(seg.begin(), seg.end());
  for (size_t i = 1; i < seg.size(); i++)
    if (seg[i - 1].first + seg[i - 1].second > seg[i].first) return false;
  return true;
}

// Word of the first id >= lo in row v of the word rows (~0u when there is none).
inline uint32_t record_word(const Words& w, uint32_t v, uint32_t lo) {
  for (uint32_t p = w.wptr[v]; p < w.wptr[v + 1]; p++) {
    const uint32_t word = w.pairs[2 * p], mask = w.pairs[2 * p + 1];
    for (uint32_t bit = 0; bit < 32; bit++)
      if ((mask >> bit & 1) && word * 32 + bit >= lo) return word;
  }
  return ~0u;
}

// `src` is the CSR the block CSR splits (the oriented graph for the forward
// tiles, its transpose for the reversed ones); `w` holds the oriented graph's
// word rows, read only for the records.  Rows >= src.n (cuts[P] may exceed n)
// must be empty.
inline std::string tiles(const char* name, const Csr& src, const Tiles& t, const Words& w) {
  const std::string pre = std::string(name) + ": ";
  const uint32_t P = t.P;
  std::vector<std::pair<uint64_t, uint64_t>> rseg, cseg, eseg;
  for (uint32_t x = 0; x < P; x++)
    for (uint32_t y = 0; y < P; y++) {
      const uint32_t id = x * P + y;
      const uint32_t H = t.cuts[x + 1] - t.cuts[x], W = t.cuts[y + 1] - t.cuts[y];
      const uint64_t ro = t.rp_off[id];
      if (ro % 4) return pre + at("row segment not 16-byte aligned, tile", id);
      if (ro + H + 1 > t.rp_len) return pre + at("row segment outside the pool, tile", id);
      rseg.push_back({ro, (uint64_t)H + 1});
      const uint32_t* r = t.rp + ro;
      if (r[0] != 0) return pre + at("row segment does not start at 0, tile", id);
      if (r[H] != t.nnz[id]) return pre + at("row segment does not end at nnz, tile", id);
      const uint64_t co = t.col_off[id];
      const uint32_t z = t.nnz[id];
      if (z == 0) {
        if (co != kNoSeg) return pre + at("empty tile has a column segment", id);
      } else {
        if (co == kNoSeg || co % 4) return pre + at("column segment missing or not 16-byte aligned, tile", id);
        if (co + z > t.col_len) return pre + at("column segment outside the pool, tile", id);
        cseg.push_back({co, z});
        const uint64_t eo = co / 32 + id, el = (z + 31) / 32;
        if (eo + el > t.erow_len) return pre + at("row index outside its pool, tile", id);
        eseg.push_back({eo, el});
      }
      uint32_t mx = 0, ne = 0;
      for (uint32_t b = 0; b < H; b++) {
        const uint32_t s = r[b], e = r[b + 1];
        if (e < s || e > z) return pre + at("row pointers decrease, tile / row", id, b);
        const uint32_t len = e - s;
        mx = len > mx ? len : mx;
        ne += len != 0;
        // the source row's ids inside column part y
        const uint32_t u = t.cuts[x] + b;
        uint32_t a0 = 0, a1 = 0;
        if (u < src.n) {
          a0 = src.indptr[u];
          a1 = src.indptr[u + 1];
          while (a0 < a1 && src.indices[a0] < t.cuts[y]) a0++;
          uint32_t k = a0;
          while (k < a1 && src.indices[k] < t.cuts[y + 1]) k++;
          a1 = k;
        }
        if (a1 - a0 != len) return pre + at("tile row length differs from the source row, tile / row", id, b);
        for (uint32_t q = 0; q < len; q++) {
          const uint32_t c = t.col[co + s + q];
          if (c >= W) return pre + at("column >= tile width, tile / row", id, b);
          if (q && t.col[co + s + q - 1] >= c) return pre + at("tile row not strictly increasing, tile / row", id, b);
        }
        for (uint32_t q = 0; q < len; q++) {
          const uint32_t c = t.col[co + s + q];
          if (c + t.cuts[y] != src.indices[a0 + q]) return pre + at("tile row differs from the source row, tile / row", id, b);
          if (t.rec) {
            // reversed entry (row v, column u) stands for forward edge u -> v
            const uint32_t v = u, fu = c + t.cuts[y];
            const uint32_t p0 = t.rec[2 * (co + s + q)], p1 = t.rec[2 * (co + s + q) + 1];
            if (p1 != w.wptr[fu + 1] || p0 < w.wptr[fu] || p0 >= p1)
              return pre + at("record outside the row's pairs, tile / row", id, b);
            const uint32_t lw = record_word(w, v, t.cuts[x]);
            if (lw < v / 32) {
              if (w.pairs[2 * p0] < lw || (p0 > w.wptr[fu] && w.pairs[2 * (p0 - 1)] >= lw))
                return pre + at("record names the wrong pair, tile / row", id, b);
            } else if (w.pairs[2 * p0] != v / 32 || !(w.pairs[2 * p0 + 1] >> (v % 32) & 1)) {
              return pre + at("record names the wrong pair, tile / row", id, b);
            }
          }
        }
        for (uint32_t q = (s + 31) & ~31u; q < e; q += 32)
          if (t.erow[co / 32 + id + q / 32] != b) return pre + at("row index names the wrong row, tile / entry", id, q);
      }
      if (mx != t.maxdeg[id]) return pre + at("longest row differs, tile", id);
      if (ne != t.nerows[id]) return pre + at("non-empty row count differs, tile", id);
    }
  if (!disjoint(rseg)) return pre + "row segments overlap";
  if (!disjoint(cseg)) return pre + "column segments overlap";
  if (!disjoint(eseg)) return pre + "row index segments overlap";
  return "";
}

}  // namespace check
}  // namespace bbtc

// Test program for bbtc_b200/csrc/layout_check.hpp: builds the block-CSR
// layout of a graph on the host, in the format the device builder writes
// (bbtc_b200/csrc/layout.cu), plants one named fault in it and prints what
// the checker says ("OK" when it finds nothing).
//
// usage: layout_check_harness <graph file> <fault>
// graph file: uint32 n, uint32 P, uint64 m, indptr[n+1], indices[m], cuts[P+1]
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "layout_check.hpp"

using namespace bbtc::check;

struct Built {
  std::vector<uint64_t> rp_off, col_off;
  std::vector<uint32_t> nnz, maxdeg, nerows, rp, col, erow, rec;
};

static uint64_t align4(uint64_t x) { return (x + 3) & ~3ull; }

// One block CSR of `src` over the cuts; with `w` (and the oriented CSR `fwd`),
// the records of the reversed tiles.
static Built build(const Csr& src, uint32_t P, const std::vector<uint32_t>& cuts, const Words* w,
                   const Csr* fwd = nullptr) {
  const uint32_t T = P * P;
  Built b;
  b.rp_off.assign(T, 0);
  uint64_t cur = 0;
  for (uint32_t x = 0; x < P; x++) {
    const uint64_t A = align4((uint64_t)cuts[x + 1] - cuts[x] + 1);
    for (uint32_t y = 0; y < P; y++) b.rp_off[x * P + y] = cur + y * A;
    cur += A * P;
  }
  b.rp.assign(cur + 4, 0);
  b.nnz.assign(T, 0);
  b.maxdeg.assign(T, 0);
  b.nerows.assign(T, 0);
  auto seg = [&](uint32_t u, uint32_t y, uint32_t& a0, uint32_t& a1) {
    a0 = a1 = 0;
    if (u >= src.n) return;
    a0 = src.indptr[u];
    a1 = src.indptr[u + 1];
    while (a0 < a1 && src.indices[a0] < cuts[y]) a0++;
    uint32_t k = a0;
    while (k < a1 && src.indices[k] < cuts[y + 1]) k++;
    a1 = k;
  };
  for (uint32_t x = 0; x < P; x++)
    for (uint32_t y = 0; y < P; y++) {
      const uint32_t t = x * P + y;
      uint32_t* r = &b.rp[b.rp_off[t]];
      for (uint32_t i = 0; i < cuts[x + 1] - cuts[x]; i++) {
        uint32_t a0, a1;
        seg(cuts[x] + i, y, a0, a1);
        r[i + 1] = r[i] + (a1 - a0);
        b.maxdeg[t] = std::max(b.maxdeg[t], a1 - a0);
        b.nerows[t] += a1 > a0;
      }
      b.nnz[t] = r[cuts[x + 1] - cuts[x]];
    }
  b.col_off.assign(T, kNoSeg);
  cur = 0;
  for (uint32_t t = 0; t < T; t++) {
    if (b.nnz[t]) b.col_off[t] = cur;
    cur += align4(b.nnz[t]);
  }
  const uint64_t col_len = src.m + 4ull * T + 4;
  b.col.assign(col_len, 0);
  b.erow.assign(col_len / 32 + T + 1, 0xdeadbeefu);
  if (w) b.rec.assign(2 * col_len, 0);
  for (uint32_t x = 0; x < P; x++)
    for (uint32_t y = 0; y < P; y++) {
      const uint32_t t = x * P + y;
      if (!b.nnz[t]) continue;
      const uint32_t* r = &b.rp[b.rp_off[t]];
      for (uint32_t i = 0; i < cuts[x + 1] - cuts[x]; i++) {
        uint32_t a0, a1;
        seg(cuts[x] + i, y, a0, a1);
        for (uint32_t q = 0; q < a1 - a0; q++) {
          const uint64_t pos = b.col_off[t] + r[i] + q;
          const uint32_t c = src.indices[a0 + q];
          b.col[pos] = c - cuts[y];
          if (w) {
            // reversed entry (v, u): the pair of row u holding v -- or, when v's
            // row has its first id >= cuts[x] in a lower word, the first pair
            // of row u at or above that word -- and row u's pair end
            const uint32_t v = cuts[x] + i;
            uint32_t lw = v / 32;
            if (fwd) {
              // first id of v's oriented row at or above cuts[x]
              uint32_t k = fwd->indptr[v];
              while (k < fwd->indptr[v + 1] && fwd->indices[k] < cuts[x]) k++;
              if (k < fwd->indptr[v + 1] && fwd->indices[k] / 32 < lw) lw = fwd->indices[k] / 32;
            }
            uint32_t p = w->wptr[c];
            while (w->pairs[2 * p] < lw) p++;
            b.rec[2 * pos] = p;
            b.rec[2 * pos + 1] = w->wptr[c + 1];
          }
        }
        for (uint32_t q = (r[i] + 31) & ~31u; q < r[i + 1]; q += 32) b.erow[b.col_off[t] / 32 + t + q / 32] = i;
      }
    }
  return b;
}

static Tiles view(const Built& b, uint32_t P, const std::vector<uint32_t>& cuts) {
  Tiles t;
  t.P = P;
  t.cuts = cuts.data();
  t.rp_off = b.rp_off.data();
  t.col_off = b.col_off.data();
  t.nnz = b.nnz.data();
  t.maxdeg = b.maxdeg.data();
  t.nerows = b.nerows.data();
  t.rp = b.rp.data();
  t.rp_len = b.rp.size();
  t.col = b.col.data();
  t.col_len = b.col.size();
  t.erow = b.erow.data();
  t.erow_len = b.erow.size();
  t.rec = b.rec.empty() ? nullptr : b.rec.data();
  return t;
}

// first non-empty tile with a row of at least `len` entries: (tile, row)
static bool find_row(const Built& b, uint32_t P, const std::vector<uint32_t>& cuts, uint32_t len, uint32_t& t,
                     uint32_t& row) {
  for (t = 0; t < P * P; t++) {
    const uint32_t H = cuts[t / P + 1] - cuts[t / P];
    const uint32_t* r = &b.rp[b.rp_off[t]];
    for (row = 0; row < H; row++)
      if (r[row + 1] - r[row] >= len) return true;
  }
  return false;
}

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 2;
  uint32_t n = 0, P = 0;
  uint64_t m = 0;
  bool ok = std::fread(&n, 4, 1, f) == 1 && std::fread(&P, 4, 1, f) == 1 && std::fread(&m, 8, 1, f) == 1;
  std::vector<uint32_t> indptr((size_t)n + 1), indices(m), cuts(P + 1);
  ok = ok && std::fread(indptr.data(), 4, n + 1, f) == n + 1;
  ok = ok && (m == 0 || std::fread(indices.data(), 4, m, f) == m);
  ok = ok && std::fread(cuts.data(), 4, P + 1, f) == P + 1;
  std::fclose(f);
  if (!ok) return 2;
  const std::string fault = argv[2];

  // word-compressed rows
  std::vector<uint32_t> wptr((size_t)n + 1, 0), pairs;
  for (uint32_t u = 0; u < n; u++) {
    for (uint32_t e = indptr[u]; e < indptr[u + 1]; e++) {
      const uint32_t word = indices[e] / 32;
      if (e == indptr[u] || indices[e - 1] / 32 != word) {
        pairs.push_back(word);
        pairs.push_back(0);
      }
      pairs.back() |= 1u << (indices[e] % 32);
    }
    wptr[u + 1] = (uint32_t)(pairs.size() / 2);
  }
  pairs.resize(2 * std::max<uint64_t>(m, 1), 0);
  Csr g{n, m, indptr.data(), indices.data()};
  Words w{wptr.data(), pairs.data(), std::max<uint64_t>(m, 1)};
  std::vector<uint32_t> tp, tc;
  transpose(g, tp, tc);
  Csr tr{n, m, tp.data(), tc.data()};
  Built fwd = build(g, P, cuts, nullptr);
  Built rev = build(tr, P, cuts, &w, &g);
  // pivot descriptors: row start, pair start, first id, last id
  std::vector<uint32_t> desc(4 * ((size_t)n + 1), 0);
  for (uint32_t u = 0; u <= n; u++) {
    desc[4 * u] = indptr[u];
    desc[4 * u + 1] = wptr[u];
    if (u < n && indptr[u + 1] > indptr[u]) {
      desc[4 * u + 2] = indices[indptr[u]];
      desc[4 * u + 3] = indices[indptr[u + 1] - 1];
    }
  }

  uint32_t t = 0, row = 0;
  auto entry = [&](Built& b, uint32_t len) -> uint64_t {
    if (!find_row(b, P, cuts, len, t, row)) {
      std::printf("NO-SITE\n");
      std::exit(3);
    }
    return b.col_off[t] + b.rp[b.rp_off[t] + row];
  };
  if (fault == "none") {
  } else if (fault == "csr_unsorted") {
    for (uint32_t u = 0; u < n; u++)
      if (indptr[u + 1] - indptr[u] >= 2) {
        std::swap(indices[indptr[u]], indices[indptr[u] + 1]);
        break;
      }
  } else if (fault == "word_mask") {
    pairs[1] = 0;
  } else if (fault == "word_order") {
    for (uint32_t u = 0; u < n; u++)
      if (wptr[u + 1] - wptr[u] >= 2) {
        std::swap(pairs[2 * wptr[u]], pairs[2 * wptr[u] + 2]);
        std::swap(pairs[2 * wptr[u] + 1], pairs[2 * wptr[u] + 3]);
        break;
      }
  } else if (fault == "rp_misaligned") {
    fwd.rp_off[1] += 1;
  } else if (fault == "rp_nnz") {
    entry(fwd, 1);
    fwd.nnz[t] += 1;
  } else if (fault == "col_misaligned") {
    entry(fwd, 1);
    fwd.col_off[t] += 2;
  } else if (fault == "col_empty_segment") {
    for (t = 0; t < P * P && fwd.nnz[t]; t++) {
    }
    if (t == P * P) {
      std::printf("NO-SITE\n");
      return 3;
    }
    fwd.col_off[t] = 0;
  } else if (fault == "col_width") {
    const uint64_t p = entry(fwd, 1);
    fwd.col[p] = cuts[t % P + 1] - cuts[t % P];
  } else if (fault == "col_swap") {
    const uint64_t p = entry(fwd, 2);
    std::swap(fwd.col[p], fwd.col[p + 1]);
  } else if (fault == "col_value") {
    const uint64_t p = entry(fwd, 1);
    const uint32_t W = cuts[t % P + 1] - cuts[t % P];
    const uint32_t len = fwd.rp[fwd.rp_off[t] + row + 1] - fwd.rp[fwd.rp_off[t] + row];
    // move the row's last column to a free slot above it (or below its first)
    uint32_t& last = fwd.col[p + len - 1];
    if (last + 1 < W) last += 1;
    else if (fwd.col[p] > 0) fwd.col[p] -= 1;
    else {
      std::printf("NO-SITE\n");
      return 3;
    }
  } else if (fault == "maxdeg") {
    entry(fwd, 1);
    fwd.maxdeg[t] += 1;
  } else if (fault == "nerows") {
    entry(fwd, 1);
    fwd.nerows[t] += 1;
  } else if (fault == "erow") {
    entry(rev, 1);
    rev.erow[rev.col_off[t] / 32 + t] ^= 1;
  } else if (fault == "rec_pair") {
    const uint64_t p = entry(rev, 1);
    rev.rec[2 * p] += 1;
  } else if (fault == "rec_end") {
    const uint64_t p = entry(rev, 1);
    rev.rec[2 * p + 1] += 1;
  } else if (fault == "desc_last") {
    for (uint32_t u = 0; u < n; u++)
      if (indptr[u + 1] > indptr[u]) {
        desc[4 * u + 3] += 1;
        break;
      }
  } else {
    return 2;
  }

  std::string why = csr(g);
  if (why.empty()) why = words(g, w);
  if (why.empty()) why = descs(g, w, desc.data());
  if (why.empty()) why = tiles("reversed tiles", tr, view(rev, P, cuts), w);
  if (why.empty()) why = tiles("forward tiles", g, view(fwd, P, cuts), w);
  std::printf("%s\n", why.empty() ? "OK" : why.c_str());
  return 0;
}

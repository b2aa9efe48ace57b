// Graph files for the drop-in CLI: edge lists, MatrixMarket coordinate files
// and the `.bbtc` binary CSR cache.
//
// Formats follow the reference's reader (the vendored PIGO library):
//   * edge list: one pair of non-negative ids per line; lines starting with
//     '#' or '%' are comments; further columns (weights) are ignored
//     (PIGO pigo/impl/pigo.impl.hpp:184-186, 277-330).  Vertices = largest id + 1.
//   * MatrixMarket: "%%MatrixMarket matrix coordinate ..." header, comments,
//     a "rows cols nnz" line, then 1-based entries whose ids are kept as they
//     are, so vertex 0 is isolated (PIGO pigo/impl/coo.impl.hpp:318-330).
//   * `.bbtc`: PIGO's binary CSR, "PIGO-CSR-v2" then uint8 sizeof(label) and
//     uint8 sizeof(offset) (both 4), then n, m, nrows, ncols (uint32) and the
//     offsets[n+1] and endpoints[m] arrays (PIGO pigo/impl/csr.impl.hpp:441-513).
//     The reference stores the degree-ordered, oriented graph there after the
//     first text read (include/utils/utils.hpp:260-268) and loads it instead
//     of the text file when present (utils.hpp:168-170); so does this CLI.
// Text inputs are symmetrised, cleaned and oriented by bbtcg_from_pairs.
#include <sys/stat.h>

#include <algorithm>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

extern "C" int bbtcg_from_pairs(uint32_t n, const uint32_t* src, const uint32_t* dst, uint64_t m, void** handle);
extern "C" int bbtcg_from_csr(uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m,
                              void** handle);

namespace {

const char kMagic[] = "PIGO-CSR-v2";

bool read_file(const char* path, std::string& buf) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::fseek(f, 0, SEEK_END);
  const long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  if (sz < 0) {
    std::fclose(f);
    return false;
  }
  buf.resize((size_t)sz);
  const size_t got = sz ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
  std::fclose(f);
  return got == (size_t)sz;
}

// A cached CSR is trusted by nothing downstream (the host partitioners index
// arrays with it), so it must meet the upload contract: indptr starts at 0,
// never decreases and ends at m; every row is strictly increasing with ids < n.
bool csr_ok(uint64_t n, uint64_t m, const uint32_t* indptr, const uint32_t* indices) {
  if (indptr[0] != 0 || indptr[n] != m) return false;
  for (uint64_t u = 0; u < n; u++) {
    const uint32_t a = indptr[u], b = indptr[u + 1];
    if (b < a) return false;
    for (uint32_t e = a; e < b; e++)
      if (indices[e] >= n || (e > a && indices[e - 1] >= indices[e])) return false;
  }
  return true;
}

bool ends_with(const std::string& s, const std::string& t) {
  return s.size() >= t.size() && s.compare(s.size() - t.size(), t.size(), t) == 0;
}

// Parse pairs from text starting at `pos`; returns -1 on a malformed line.
int parse_pairs(const std::string& b, size_t pos, std::vector<uint32_t>& src, std::vector<uint32_t>& dst,
                uint64_t& maxid) {
  const size_t n = b.size();
  while (pos < n) {
    while (pos < n && (b[pos] == ' ' || b[pos] == '\t' || b[pos] == '\r' || b[pos] == '\n')) pos++;
    if (pos >= n) break;
    if (b[pos] == '#' || b[pos] == '%') {
      while (pos < n && b[pos] != '\n') pos++;
      continue;
    }
    uint64_t v[2];
    for (int k = 0; k < 2; k++) {
      while (pos < n && (b[pos] == ' ' || b[pos] == '\t')) pos++;
      if (pos >= n || !std::isdigit((unsigned char)b[pos])) return -1;
      uint64_t x = 0;
      while (pos < n && std::isdigit((unsigned char)b[pos])) {
        x = x * 10 + (uint64_t)(b[pos] - '0');
        if (x >= 0xffffffffull) return -1;
        pos++;
      }
      v[k] = x;
    }
    while (pos < n && b[pos] != '\n') pos++;  // ignore further columns
    src.push_back((uint32_t)v[0]);
    dst.push_back((uint32_t)v[1]);
    if (v[0] > maxid) maxid = v[0];
    if (v[1] > maxid) maxid = v[1];
  }
  return 0;
}

}  // namespace

extern "C" {

// Format of `path` as the reference would pick it: 2 = PIGO binary CSR (by
// magic), 1 = MatrixMarket (".mtx"), 0 = edge list.
int bbtcio_guess(const char* path) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return -1;
  char head[sizeof(kMagic)] = {0};
  const size_t got = std::fread(head, 1, sizeof(kMagic) - 1, f);
  std::fclose(f);
  if (got == sizeof(kMagic) - 1 && std::memcmp(head, kMagic, sizeof(kMagic) - 1) == 0) return 2;
  if (ends_with(path, ".mtx")) return 1;
  return 0;
}

// Read a graph file into an oriented-CSR handle (free with bbtcg_free).
// Returns 0, -1 (unreadable / malformed), -2 (out of memory), -3 (too large).
int bbtcio_read(const char* path, int* kind, void** handle) {
  if (!path || !handle) return -1;
  const int k = bbtcio_guess(path);
  if (k < 0) return -1;
  if (kind) *kind = k;
  std::string b;
  if (!read_file(path, b)) return -1;
  if (k == 2) {
    size_t off = sizeof(kMagic) - 1;
    if (b.size() < off + 2 + 16) return -1;
    const uint8_t lsz = (uint8_t)b[off], osz = (uint8_t)b[off + 1];
    off += 2;
    if (lsz != 4 || osz != 4) return -1;
    uint32_t hdr[4];
    std::memcpy(hdr, b.data() + off, sizeof(hdr));
    off += sizeof(hdr);
    const uint64_t n = hdr[0], m = hdr[1];
    if (b.size() < off + 4 * (n + 1) + 4 * m) return -1;  // truncated
    if (n >= 0xffffffffull) return -3;
    // the arrays start 30 bytes in: copy them out to aligned storage
    std::vector<uint32_t> indptr((size_t)n + 1), indices((size_t)m);
    std::memcpy(indptr.data(), b.data() + off, 4 * (n + 1));
    if (m) std::memcpy(indices.data(), b.data() + off + 4 * (n + 1), 4 * m);
    if (!csr_ok(n, m, indptr.data(), indices.data())) return -1;
    return bbtcg_from_csr((uint32_t)n, indptr.data(), indices.data(), m, handle);
  }
  std::vector<uint32_t> src, dst;
  uint64_t maxid = 0;
  size_t pos = 0;
  uint64_t nrows = 0;
  if (k == 1) {
    if (b.compare(0, 32, "%%MatrixMarket matrix coordinate") != 0) return -1;
    // skip the header and comment lines, then read "rows cols nnz"
    while (pos < b.size() && (b[pos] == '%' || b[pos] == '\n' || b[pos] == '\r')) {
      while (pos < b.size() && b[pos] != '\n') pos++;
      if (pos < b.size()) pos++;
    }
    unsigned long long r = 0, c = 0, z = 0;
    if (std::sscanf(b.c_str() + pos, "%llu %llu %llu", &r, &c, &z) != 3) return -1;
    nrows = std::max<uint64_t>(r, c) + 1;  // ids stay 1-based
    while (pos < b.size() && b[pos] != '\n') pos++;
  }
  if (parse_pairs(b, pos, src, dst, maxid) != 0) return -1;
  uint64_t n = src.empty() ? 0 : maxid + 1;
  if (nrows > n) n = nrows;
  if (n >= 0xffffffffull) return -3;
  return bbtcg_from_pairs((uint32_t)n, src.data(), dst.data(), src.size(), handle);
}

// Write the `.bbtc` cache (PIGO-CSR-v2, 32-bit labels and offsets).
int bbtcio_write_bbtc(const char* path, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m) {
  if (!path || !indptr || (m && !indices) || m >= (1ull << 32)) return -1;
  FILE* f = std::fopen(path, "wb");
  if (!f) return -1;
  const uint8_t sz[2] = {4, 4};
  const uint32_t hdr[4] = {n, (uint32_t)m, n, n};
  bool ok = std::fwrite(kMagic, 1, sizeof(kMagic) - 1, f) == sizeof(kMagic) - 1;
  ok = ok && std::fwrite(sz, 1, 2, f) == 2;
  ok = ok && std::fwrite(hdr, sizeof(uint32_t), 4, f) == 4;
  ok = ok && std::fwrite(indptr, sizeof(uint32_t), (size_t)n + 1, f) == (size_t)n + 1;
  if (m) ok = ok && std::fwrite(indices, sizeof(uint32_t), m, f) == m;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? 0 : -1;
}

}  // extern "C"

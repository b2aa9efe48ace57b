// Device-resident block-CSR layout.
//
// The reference splits the oriented CSR into P x P tile CSRs on the host:
// a per-row count by tile column, a serial exclusive scan over P*(N+P) row
// slots and a scatter of tile-local column ids
// (src/data_structures/block_csr.cpp:288-376), then copies tiles to the GPU
// lazily, one cudaMalloc + two copies + a stream sync per tile
// (src/triangle_counting/bb_tc_helper.cpp:75-110).  Here the whole layout is
// built on the device once and stays resident:
//
//   * the oriented CSR itself (global ids), which the fused task rows probe;
//   * forward tiles (x, y): rows of part x, tile-local columns of part y --
//     the reference's tiles, used as ab / bc / ac by the per-task kernels;
//   * reversed tiles (y, x): the same edges grouped by their column vertex --
//     the CSC of forward tile (x, y) -- with, beside each entry, the record
//     of its forward edge (u, v): the range of row u's word-compressed pairs
//     from the one that holds v (or, when the pivot row N+(v) has ids below
//     v inside the task columns, from the first pair that can hold one: see
//     record_start) to the row's end, which is what a fused task row streams
//     per entry;
//   * the word-compressed rows of the oriented CSR: row u's ids grouped by
//     32-id word into (word index, bit mask) pairs.
//
// Every tile owns a row-pointer segment of H+1 tile-local offsets (first
// entry 0) in one pool, laid out like the reference's rows_ array (P segments
// per row part); column segments hold only the non-empty tiles.  Segments
// start on 16-byte boundaries.  All passes are edge-parallel: each edge finds
// its tile by bisection of the cut vector and the first edge of every (row,
// tile) run writes the run length, so no thread walks a whole row.
#include <cub/cub.cuh>
#include <cuda.h>

#include <algorithm>
#include <cstring>

#include "internal.h"
#include "layout_check.hpp"

namespace bbtc {

namespace {

constexpr uint32_t FULLMASK = 0xffffffffu;

__device__ __forceinline__ uint32_t part_of(const uint32_t* cuts, uint32_t P, uint32_t u) {
  // largest x in [0, P) with cuts[x] <= u (skips empty parts); needs u < cuts[P]
  uint32_t lo = 0, hi = P;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (cuts[mid] <= u) lo = mid; else hi = mid;
  }
  return lo;
}

// first position p in [lo, hi) with a[p] >= x
__device__ __forceinline__ uint32_t lower_bound_range(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                                      uint32_t x) {
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Host-to-device copy done by the SMs: `src` is page-locked host memory
// mapped into the device's address space, read over the host link, so the
// copy does not queue behind other streams' transfers on the copy engines.
// Each `dst` is a device allocation (256-byte aligned); words = bytes / 4.
// Two arrays per launch (a graph's row pointers and ids); words1 may be 0.
__device__ __forceinline__ void copy_words(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                                           uint64_t words, uint64_t t0, uint64_t stride) {
  uint64_t done = 0;
  if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
    const uint64_t v = words / 4;
    const uint4* __restrict__ s4 = reinterpret_cast<const uint4*>(src);
    uint4* __restrict__ d4 = reinterpret_cast<uint4*>(dst);
    for (uint64_t i = t0; i < v; i += stride) d4[i] = s4[i];
    done = v * 4;
  }
  for (uint64_t i = done + t0; i < words; i += stride) dst[i] = src[i];
}

__global__ void k_copy_mapped(uint32_t* __restrict__ dst0, const uint32_t* __restrict__ src0, uint64_t words0,
                              uint32_t* __restrict__ dst1, const uint32_t* __restrict__ src1, uint64_t words1) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  copy_words(dst0, src0, words0, t0, stride);
  copy_words(dst1, src1, words1, t0, stride);
}

// Input contract check and per-edge expansion, one warp per row: row
// pointers start at 0, never decrease and end at m; rows are strictly
// increasing; ids are < n.  Rows whose pointers are out of order or past m
// are flagged and skipped.  Writes the row id of every edge; with `flags`,
// marks the edges that open a new 32-id word of their row (flags[e] = 1), the
// input of the word-compressed rows; with `iota`, iota[e] = e (the edge ids
// that the reversed graph's sort carries).  Nothing downstream reads `bad`
// on the host before the layout is done: every later kernel that indexes by
// these arrays returns at once when `*bad` is set.
__global__ void k_expand_check(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                               uint32_t n, uint64_t m, uint32_t* __restrict__ rows, uint32_t* __restrict__ bad,
                               uint32_t* __restrict__ flags, uint32_t* __restrict__ iota) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < n; u += nwarps) {
    const uint32_t a = indptr[u], b = indptr[u + 1];
    if (lane == 0) {
      if (u == 0 && a != 0) atomicOr(bad, 1u);
      if (u == n - 1 && (uint64_t)b != m) atomicOr(bad, 2u);
    }
    if (b < a || (uint64_t)b > m) {
      if (lane == 0) atomicOr(bad, 4u);
      continue;
    }
    for (uint32_t e = a + lane; e < b; e += 32) {
      rows[e] = u;
      const uint32_t c = indices[e];
      const uint32_t prev = e > a ? indices[e - 1] : 0u;
      if (c >= n) atomicOr(bad, 8u);
      if (e > a && prev >= c) atomicOr(bad, 16u);
      if (flags) flags[e] = (e == a || (c >> 5) != (prev >> 5)) ? 1u : 0u;
      if (iota) iota[e] = e;
    }
  }
}

// Run lengths: the first edge of each (row, tile) run writes the length into
// slot (rp_off[tile] + local row + 1) of the counts buffer.  runs[e] = e for
// the first edge of a run, else 0: its inclusive max-scan gives every edge
// the start of its run.
__global__ void k_entry_count(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                              const uint32_t* __restrict__ rows, uint64_t m, const uint32_t* __restrict__ cuts_g,
                              uint32_t P, const uint64_t* __restrict__ rp_off, uint32_t* __restrict__ counts,
                              uint32_t* __restrict__ runs, const uint32_t* __restrict__ bad) {
  if (*bad) return;
  __shared__ uint32_t cuts[kMaxParts + 1];
  for (uint32_t t = threadIdx.x; t <= P; t += blockDim.x) cuts[t] = cuts_g[t];
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint32_t u = rows[e];
    const uint32_t c = indices[e];
    const uint32_t y = part_of(cuts, P, c);
    const uint32_t a = indptr[u];
    const bool first = e == a || indices[e - 1] < cuts[y];
    runs[e] = first ? (uint32_t)e : 0u;
    if (!first) continue;
    const uint32_t end = lower_bound_range(indices, (uint32_t)e, indptr[u + 1], cuts[y + 1]);
    const uint32_t x = part_of(cuts, P, u);
    counts[rp_off[x * P + y] + (u - cuts[x]) + 1] = end - (uint32_t)e;
  }
}

// Up to four zero fills of layout buffers in one launch, on the SMs (at the
// stream's priority, leaving the copy engines to the uploads); each range
// starts on a 16-byte boundary.
struct ZeroRanges {
  uint32_t* p[4];
  uint64_t words[4];
};

__global__ void k_zero_ranges(ZeroRanges z) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int r = 0; r < 4; r++) {
    uint32_t* __restrict__ p = z.p[r];
    const uint64_t nwords = z.words[r];
    uint4* __restrict__ q = reinterpret_cast<uint4*>(p);
    const uint64_t n4 = nwords / 4;
    for (uint64_t i = t0; i < n4; i += stride) q[i] = make_uint4(0, 0, 0, 0);
    for (uint64_t i = n4 * 4 + t0; i < nwords; i += stride) p[i] = 0;
  }
}

// One pass over the row-pointer pool: `scanned` is the inclusive scan of the
// run counts, so a slot minus its tile's first slot is the tile-local row
// pointer written to `rp`; per tile, the longest row and the number of
// non-empty rows (a row's length is the difference of two scanned slots).
// Lanes of one tile are combined before the atomics.
__global__ void k_localize_stats(uint32_t* __restrict__ rp, const uint32_t* __restrict__ scanned,
                                 const uint32_t* __restrict__ cuts_g, uint32_t P,
                                 const uint64_t* __restrict__ part_off, uint64_t len, uint32_t* __restrict__ maxdeg,
                                 uint32_t* __restrict__ nerows, const uint32_t* __restrict__ bad) {
  if (*bad) return;
  __shared__ uint32_t cuts[kMaxParts + 1];
  __shared__ uint64_t poff[kMaxParts + 1];
  for (uint32_t t = threadIdx.x; t <= P; t += blockDim.x) {
    cuts[t] = cuts_g[t];
    poff[t] = part_off[t];
  }
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t start = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t iters = (len + stride - 1) / stride;  // the same for every lane of a warp
  for (uint64_t it = 0; it < iters; it++) {
    const uint64_t s = start + it * stride;
    uint32_t tile = 0xffffffffu, rowlen = 0;
    if (s < len) {
      uint32_t lo = 0, hi = P;  // row part x: last x with part_off[x] <= s
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (poff[mid] <= s) lo = mid; else hi = mid;
      }
      const uint64_t A = (poff[lo + 1] - poff[lo]) / P;  // slots per tile of this row part
      const uint32_t y = (uint32_t)((s - poff[lo]) / A);
      const uint32_t r = (uint32_t)(s - poff[lo] - (uint64_t)y * A);
      const uint32_t v = scanned[s];
      rp[s] = v - scanned[poff[lo] + (uint64_t)y * A];
      if (r < cuts[lo + 1] - cuts[lo]) {
        rowlen = scanned[s + 1] - v;
        tile = lo * P + y;
      }
    }
    // a warp's 32 slots lie in one tile but at a tile's end: group lanes by
    // tile only there (match and a per-group reduction are slow)
    const uint32_t grp = __all_sync(FULLMASK, tile == __shfl_sync(FULLMASK, tile, 0))
                             ? FULLMASK
                             : __match_any_sync(FULLMASK, tile);
    const uint32_t mx = __reduce_max_sync(grp, rowlen);
    const uint32_t ne = __popc(grp & __ballot_sync(FULLMASK, rowlen != 0));
    if (tile != 0xffffffffu && lane == (uint32_t)(__ffs(grp) - 1)) {
      if (ne) atomicAdd(&nerows[tile], ne);
      if (mx) atomicMax(&maxdeg[tile], mx);
    }
  }
}

// nnz per tile and 16-byte aligned column offsets of the non-empty tiles:
// one warp, 32 tiles at a time, an exclusive scan of the aligned sizes by
// shuffles (launched as one block of 32 threads).
__global__ void k_tile_offsets(const uint32_t* __restrict__ rp, const uint64_t* __restrict__ rp_off,
                               const uint32_t* __restrict__ cuts, uint32_t P, uint32_t* __restrict__ nnz,
                               uint64_t* __restrict__ col_off, const uint32_t* __restrict__ bad) {
  if (blockIdx.x != 0 || threadIdx.x >= 32 || *bad) return;
  const uint32_t lane = threadIdx.x;
  const uint32_t T = P * P;
  uint64_t cur = 0;
  for (uint32_t t0 = 0; t0 < T; t0 += 32) {
    const uint32_t t = t0 + lane;
    uint32_t z = 0;
    if (t < T) {
      const uint32_t x = t / P;
      z = rp[rp_off[t] + (cuts[x + 1] - cuts[x])];
    }
    const uint64_t size = ((uint64_t)z + 3) & ~3ull;
    uint64_t incl = size;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint64_t o = __shfl_up_sync(FULLMASK, incl, d);
      if (lane >= d) incl += o;
    }
    if (t < T) {
      nnz[t] = z;
      col_off[t] = z ? cur + incl - size : kNoSegment;
    }
    cur += __shfl_sync(FULLMASK, incl, 31);
  }
}

// Row index of every 32nd entry: erow[t][x / 32] = the row holding entry x
// of tile t, for x = 0, 32, 64, ... < nnz.  A work unit starting at a
// multiple of 32 finds its first row with one load.  Every such x lies in
// exactly one non-empty row, so each slot has one writer.  blockIdx.y = tile.
__global__ void k_row_index(const uint32_t* __restrict__ rp, const uint64_t* __restrict__ rp_off,
                            const uint32_t* __restrict__ cuts, uint32_t P, const uint64_t* __restrict__ col_off,
                            uint32_t* __restrict__ erow, const uint32_t* __restrict__ bad) {
  const uint32_t t = blockIdx.y;
  if (*bad || col_off[t] == kNoSegment) return;
  const uint32_t x = t / P;
  const uint32_t H = cuts[x + 1] - cuts[x];
  const uint32_t* __restrict__ r = rp + rp_off[t];
  uint32_t* __restrict__ er = erow + col_off[t] / 32 + t;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < H; b += gridDim.x * blockDim.x) {
    const uint32_t s = r[b], e = r[b + 1];
    // 64-bit: rounding s up to a multiple of 32 must not wrap near 2^32
    for (uint64_t q = ((uint64_t)s + 31) & ~31ull; q < e; q += 32) er[q >> 5] = b;
  }
}

// First pair of a reversed entry's record.  The entry (row v of part x,
// column c) stands for forward edge c -> v; the tasks (i, x, k >= x) count the
// common neighbours w of c and v with w >= cuts[x] (the reference's tiles
// ac = (i, k), bc = (x, k), src/triangle_counting/gpu_sparse_kernel.cu:25-46).
// The pivot side of v keeps only N+(v) ∩ [cuts[x], ∞), whose first id is L;
// the streamed side is row c from the first pair whose word can hold an id
// >= L.  When L lies in v's word or above -- always for a CSR oriented from
// lower to higher ids, where every id of N+(v) exceeds v -- that is the pair
// holding v itself (`p`); otherwise the pair is searched in row c's pairs
// before p.  Any CSR that meets the input contract counts the reference's
// task sum this way.
__device__ __forceinline__ uint32_t record_start(const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fidx,
                                                 const uint2* __restrict__ words, const uint32_t* __restrict__ wptr,
                                                 uint32_t v, uint32_t c, uint32_t lo, uint32_t p) {
  const uint32_t a = fptr[v], b = fptr[v + 1];
  if (a >= b) return p;  // no pivot: the kernel skips the row
  uint32_t L = fidx[a];
  if (L < lo) {
    const uint32_t k = lower_bound_range(fidx, a, b, lo);
    if (k >= b) return p;  // no pivot id in the task columns
    L = fidx[k];
  }
  const uint32_t lw = L >> 5;
  if (lw >= (v >> 5)) return p;
  uint32_t lo_p = wptr[c], hi_p = p;  // row c holds v, so the answer is at or before p
  while (lo_p < hi_p) {
    const uint32_t mid = lo_p + ((hi_p - lo_p) >> 1);
    if (words[mid].x < lw) lo_p = mid + 1; else hi_p = mid;
  }
  return lo_p;
}

// Scatter tile-local column ids (and, for the reversed graph, the records of
// the forward edges) into the column pool.  For the reversed graph
// `fptr` / `fidx` / `words` are the oriented CSR and its word-compressed rows.
__global__ void k_entry_scatter(const uint32_t* __restrict__ runs, const uint32_t* __restrict__ indices,
                                const uint32_t* __restrict__ rows, uint64_t m, const uint32_t* __restrict__ cuts_g,
                                uint32_t P, const uint64_t* __restrict__ rp_off, const uint64_t* __restrict__ col_off,
                                const uint32_t* __restrict__ rp, uint32_t* __restrict__ col,
                                const uint32_t* __restrict__ eids, const uint32_t* __restrict__ wpos,
                                const uint32_t* __restrict__ wptr, uint2* __restrict__ rec,
                                const uint32_t* __restrict__ fptr, const uint32_t* __restrict__ fidx,
                                const uint2* __restrict__ words, const uint32_t* __restrict__ bad) {
  if (*bad) return;
  __shared__ uint32_t cuts[kMaxParts + 1];
  for (uint32_t t = threadIdx.x; t <= P; t += blockDim.x) cuts[t] = cuts_g[t];
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint32_t u = rows[e];
    const uint32_t c = indices[e];
    const uint32_t y = part_of(cuts, P, c);
    const uint32_t x = part_of(cuts, P, u);
    const uint32_t t = x * P + y;
    const uint32_t run = runs[e];  // first edge of this (row, tile) run
    const uint64_t pos = col_off[t] + rp[rp_off[t] + (u - cuts[x])] + ((uint32_t)e - run);
    col[pos] = c - cuts[y];
    if (rec) {
      // forward edge fe = (c -> u) of this reversed entry: the pairs of row c
      // from the record's first pair to the row's end
      const uint32_t fe = eids[e];
      rec[pos] = make_uint2(record_start(fptr, fidx, words, wptr, u, c, cuts[x], wpos[fe] - 1u), wptr[c + 1]);
    }
  }
}

// Word-compressed rows: each row's ids grouped by 32-id word into (word, bit
// mask) pairs.  flags[e] = 1 when edge e opens a new word of its row
// (k_expand_check); wpos = their inclusive scan, so edge e lands in pair
// wpos[e] - 1.  A warp takes 32 consecutive edges; a pair's edges are
// consecutive, so a segmented suffix OR by shuffles (five steps, no
// divergence) gives the first lane of each pair in the chunk the bits of the
// pair's edges in the chunk.  The lane of the edge that opens a pair stores
// it, after ORing in the bits of its edges past the chunk (at most 31 more,
// only for the chunk's last pair); a pair that opened in an earlier chunk is
// that chunk's to store.  So each pair has one writer and no atomics.  Pairs
// W = wpos[m - 1] .. m + 1 (the array's unused tail) are zeroed.  Needs m > 0.
__global__ void k_word_fill(const uint32_t* __restrict__ indices, const uint32_t* __restrict__ flags,
                            const uint32_t* __restrict__ wpos, uint64_t m, uint2* __restrict__ words,
                            const uint32_t* __restrict__ bad) {
  if (*bad) return;
  const uint64_t W = wpos[m - 1];
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;  // a multiple of 32: warps keep their chunks aligned
  for (uint64_t e = t0; e - lane < m; e += stride) {
    const bool valid = e < m;
    const uint32_t x = valid ? indices[e] : 0u;
    const uint32_t p = valid ? wpos[e] - 1u : 0xffffffffu;
    uint32_t v = valid ? 1u << (x & 31) : 0u;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t o = __shfl_down_sync(FULLMASK, v, d);
      const uint32_t po = __shfl_down_sync(FULLMASK, p, d);
      if (lane + d < 32 && po == p) v |= o;
    }
    const uint32_t p_prev = __shfl_up_sync(FULLMASK, p, 1);
    const uint32_t p_last = __shfl_sync(FULLMASK, p, 31);
    if (!valid) continue;
    if (e >= W) words[e] = make_uint2(0, 0);
    if ((lane > 0 && p_prev == p) || !flags[e]) continue;  // not the opening edge of its pair
    if (p_last == p) {  // the pair reaches the chunk's last edge: it may go on past the chunk
      for (uint64_t k = e - lane + 32; k < m && !flags[k]; k++) v |= 1u << (indices[k] & 31);
    }
    words[p] = make_uint2(x >> 5, v);
  }
  if (t0 < 2) words[m + t0] = make_uint2(0, 0);
}

// wptr[u] = first pair of row u (u in [0, n]); a row's first edge opens a pair.
// desc[u]: the fused kernel's view of row u as a pivot, in one 16-byte load.
__global__ void k_word_rowptr(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                              const uint32_t* __restrict__ wpos, uint32_t n, uint64_t m, uint32_t* __restrict__ wptr,
                              uint4* __restrict__ desc, const uint32_t* __restrict__ bad) {
  if (*bad) return;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u <= n; u += gridDim.x * blockDim.x) {
    const uint32_t e = indptr[u];
    const uint32_t w = (uint64_t)e < m ? wpos[e] - 1u : (m ? wpos[m - 1] : 0u);
    wptr[u] = w;
    // pivot descriptor: row start, pair start, first and last id (0, 0 for an empty row)
    const bool has = u < n && indptr[u + 1] > e;
    desc[u] = make_uint4(e, w, has ? indices[e] : 0u, has ? indices[indptr[u + 1] - 1] : 0u);
  }
}

// The reversed graph from the (column, forward edge id) pairs sorted by
// column, in two passes (the row pointers' searches run with the whole
// GPU's parallelism, not behind the gather in one grid-stride loop):
// rev_cols[q] = source row of forward edge eids[q] (q < m) ...
__global__ void k_gather(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ eids, uint64_t m,
                         uint32_t* __restrict__ rev_cols, const uint32_t* __restrict__ bad) {
  if (*bad) return;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) rev_cols[e] = rows[eids[e]];
}

// ... and rev_indptr[v] = first position of key v in the sorted keys (v <= n).
__global__ void k_rev_indptr(const uint32_t* __restrict__ keys, uint64_t m, uint32_t n,
                             uint32_t* __restrict__ rev_indptr, const uint32_t* __restrict__ bad) {
  if (*bad) return;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v <= n; v += stride) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if (keys[mid] < v) lo = mid + 1; else hi = mid;
    }
    rev_indptr[v] = (uint32_t)lo;
  }
}

inline uint64_t align4(uint64_t x) { return (x + 3) & ~3ull; }

// True when [p, p + bytes) lies wholly inside one page-locked host allocation
// (or registered range) that the current device reads at the same address.
// Both ends are asked of the runtime, and the allocation's extent of the
// driver; any failure, or a driver that cannot answer, means "no".
bool mapped_host_range(const void* p, size_t bytes) {
  if (!p || bytes == 0 || (reinterpret_cast<uintptr_t>(p) & 3)) return false;
  const char* last = static_cast<const char*>(p) + bytes - 1;
  for (const void* q : {p, static_cast<const void*>(last)}) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (a.type != cudaMemoryTypeHost || a.devicePointer != q) return false;
  }
  using GetAttr = CUresult (*)(void*, CUpointer_attribute, CUdeviceptr);
  static const GetAttr get = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuPointerGetAttribute", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return static_cast<GetAttr>(nullptr);
    }
    return reinterpret_cast<GetAttr>(f);
  }();
  if (!get) return false;
  CUdeviceptr start = 0;
  size_t size = 0;
  if (get(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, (CUdeviceptr)p) != CUDA_SUCCESS ||
      get(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, (CUdeviceptr)p) != CUDA_SUCCESS)
    return false;
  const uint64_t b = (uint64_t)reinterpret_cast<uintptr_t>(p);
  return size > 0 && b >= start && b + bytes <= (uint64_t)start + size;
}

// Launch of a layout kernel.  A context with `open_carveout` (the server's
// large-request loaders) asks for the largest shared-memory carveout: an
// SM's split between L1 and shared memory changes only when the SM is idle,
// and a layout kernel (little shared memory of its own) otherwise runs with
// a small carveout, so while one of its blocks holds an SM -- a large
// graph's grid-stride pass runs a millisecond or more -- no block that needs
// more shared memory (a CUB scan or sort pass of a small request's layout, a
// count kernel) can start there, even from a higher-priority stream.  Other
// contexts keep the driver's choice, which leaves the passes their L1
// (R-MAT s22's layout is 2.8 ms slower with the largest carveout).
template <typename... KArgs, typename... Args>
int launch_layout(const bbtc_ctx* ctx, void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                  Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  if (ctx->open_carveout) {
    attr[0].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
    attr[0].val.sharedMemCarveout = cudaSharedmemCarveoutMaxShared;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  BBTC_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  return BBTC_OK;
}

// Build one block CSR (forward or reversed) from a CSR in device memory whose
// per-edge row ids are `rows`.  With `eids` the reversed build also writes the
// forward-edge records.  The tile statistics land in `st` (device, 4*P*P words)
// and are copied to the host by the caller.
int build_block(bbtc_ctx* ctx, BlockTiles& bt, const uint32_t* d_indptr, const uint32_t* d_indices,
                const uint32_t* d_rows, uint32_t n, uint64_t m, const std::vector<uint32_t>& cuts,
                const uint32_t* d_cuts, const uint32_t* eids, const uint32_t* wpos, const uint32_t* wptr,
                const uint32_t* fptr, const uint32_t* fidx, const uint2* words, uint32_t* d_stats,
                uint64_t* d_coloff, const uint32_t* d_bad, int grid) {
  const uint32_t P = (uint32_t)cuts.size() - 1;
  const uint32_t T = P * P;
  cudaStream_t s = ctx->stream;
  bt.P = P;
  bt.rp_off.assign(T, 0);
  std::vector<uint64_t> part_off(P + 1, 0);
  uint64_t cur = 0;
  for (uint32_t x = 0; x < P; x++) {
    part_off[x] = cur;
    const uint64_t A = align4((uint64_t)cuts[x + 1] - cuts[x] + 1);
    for (uint32_t y = 0; y < P; y++) bt.rp_off[x * P + y] = cur + y * A;
    cur += A * P;
  }
  part_off[P] = cur;
  bt.rp_len = cur + 4;  // a 16-byte tail keeps rounded-up reads inside the pool
  bt.col_len = m + 4ull * T + 4;
  bt.erow_len = bt.col_len / 32 + T + 1;  // tile t's index starts at col_off[t] / 32 + t
  {
    cudaError_t e1 = dev_malloc(&bt.d_rp, bt.rp_len * sizeof(uint32_t), s);
    cudaError_t e2 = dev_malloc(&bt.d_col, bt.col_len * sizeof(uint32_t), s);
    cudaError_t e3 = eids ? dev_malloc(&bt.d_rec, bt.col_len * sizeof(uint2), s) : cudaSuccess;
    cudaError_t e4 = dev_malloc(&bt.d_erow, bt.erow_len * sizeof(uint32_t), s);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess) {
      cudaGetLastError();
      bt.release(s);
      return fail(BBTC_ERR_NOMEM, "device allocation of the block-CSR pools failed");
    }
  }
  bt.stream = s;
  DevBuf offs, counts, runs;
  BBTC_TRY(dalloc(runs, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(offs, (T + P + 1) * sizeof(uint64_t), s));
  BBTC_TRY(dalloc(counts, bt.rp_len * sizeof(uint32_t), s));
  uint64_t* d_rp_off = offs.as<uint64_t>();
  uint64_t* d_part_off = d_rp_off + T;
  {
    // through this block CSR's own pinned region: it is not written again before the build's final sync
    uint64_t* h = reinterpret_cast<uint64_t*>(ctx->h_stage + kStageOff[eids ? 1 : 0]);
    std::memcpy(h, bt.rp_off.data(), T * sizeof(uint64_t));
    std::memcpy(h + T, part_off.data(), (P + 1) * sizeof(uint64_t));
    BBTC_CUDA(cudaMemcpyAsync(d_rp_off, h, (T + P + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  }
  {
    // run counts, column pool, tile statistics and the row-pointer pool's
    // 16-byte tail (every other slot of the pool is written below)
    ZeroRanges z{{counts.as<uint32_t>(), bt.d_col, d_stats, bt.d_rp + part_off[P]},
                 {bt.rp_len, bt.col_len, 4ull * T, bt.rp_len - part_off[P]}};
    BBTC_TRY(launch_layout(ctx, k_zero_ranges, grid, 256, s, z));
  }
  if (m > 0) {
    BBTC_TRY(launch_layout(ctx, k_entry_count, grid, 256, s, d_indptr, d_indices, d_rows, m, d_cuts, P, d_rp_off,
                           counts.as<uint32_t>(), runs.as<uint32_t>(), d_bad));
    size_t rb = 0;
    BBTC_CUDA(cub::DeviceScan::InclusiveScan(nullptr, rb, runs.as<uint32_t>(), runs.as<uint32_t>(), cub::Max(),
                                             (int64_t)m, s));
    DevBuf rtmp;
    BBTC_TRY(dalloc(rtmp, rb, s));
    BBTC_CUDA(cub::DeviceScan::InclusiveScan(rtmp.p, rb, runs.as<uint32_t>(), runs.as<uint32_t>(), cub::Max(),
                                             (int64_t)m, s));
  }
  // run counts -> their inclusive scan, in place: k_localize_stats turns it into tile-local row pointers
  size_t tmp_bytes = 0;
  BBTC_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, counts.as<uint32_t>(), counts.as<uint32_t>(),
                                          (int64_t)part_off[P], s));
  DevBuf tmp;
  BBTC_TRY(dalloc(tmp, tmp_bytes, s));
  BBTC_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmp_bytes, counts.as<uint32_t>(), counts.as<uint32_t>(),
                                          (int64_t)part_off[P], s));
  uint32_t* st_nnz = d_stats;
  uint32_t* st_max = d_stats + T;
  uint32_t* st_ne = d_stats + 2 * T;
  BBTC_TRY(launch_layout(ctx, k_localize_stats, grid, 256, s, bt.d_rp, counts.as<uint32_t>(), d_cuts, P, d_part_off,
                         part_off[P], st_max, st_ne, d_bad));
  BBTC_TRY(launch_layout(ctx, k_tile_offsets, 1, 32, s, bt.d_rp, d_rp_off, d_cuts, P, st_nnz, d_coloff, d_bad));
  {
    uint32_t maxH = 1;
    for (uint32_t x = 0; x < P; x++) maxH = std::max(maxH, cuts[x + 1] - cuts[x]);
    const uint32_t gx = std::min<uint32_t>(64, (maxH + 255) / 256);
    BBTC_TRY(launch_layout(ctx, k_row_index, dim3(gx, T), 256, s, bt.d_rp, d_rp_off, d_cuts, P, d_coloff, bt.d_erow,
                           d_bad));
  }
  if (m > 0) {
    BBTC_TRY(launch_layout(ctx, k_entry_scatter, grid, 256, s, runs.as<uint32_t>(), d_indices, d_rows, m, d_cuts, P,
                           d_rp_off, d_coloff, bt.d_rp, bt.d_col, eids, wpos, wptr,
                           reinterpret_cast<uint2*>(bt.d_rec), fptr, fidx, words, d_bad));
  }
  return BBTC_OK;
}

// Read back the tile statistics of one or two block CSRs (a may be null) with
// one sync; with `d_bad`, also the input-contract flags (into *h_bad), and
// when any is set the statistics are left unread.
int fetch_stats(bbtc_ctx* ctx, BlockTiles* a, BlockTiles& b, const uint32_t* d_stats_a, const uint64_t* d_coloff_a,
                const uint32_t* d_stats_b, const uint64_t* d_coloff_b, cudaStream_t s,
                const uint32_t* d_bad = nullptr, uint32_t* h_bad = nullptr) {
  const uint32_t T = b.P * b.P;
  // pinned staging: [coloff a | coloff b | stats a | stats b]
  uint64_t* hc = reinterpret_cast<uint64_t*>(ctx->h_stage + kStageStats);
  uint32_t* hs = reinterpret_cast<uint32_t*>(hc + 2 * T);
  if (a) {
    BBTC_CUDA(cudaMemcpyAsync(hc, d_coloff_a, T * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    BBTC_CUDA(cudaMemcpyAsync(hs, d_stats_a, 3 * T * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  }
  BBTC_CUDA(cudaMemcpyAsync(hc + T, d_coloff_b, T * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaMemcpyAsync(hs + 3 * T, d_stats_b, 3 * T * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  uint32_t* hb = reinterpret_cast<uint32_t*>(ctx->h_stage + kStageBad);
  if (d_bad) BBTC_CUDA(cudaMemcpyAsync(hb, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaStreamSynchronize(s));
  if (d_bad) {
    *h_bad = *hb;
    if (*hb) return BBTC_OK;  // the statistics are void
  }
  for (BlockTiles* p : {a, &b}) {
    if (!p) continue;
    const uint64_t* c = p == a ? hc : hc + T;
    const uint32_t* h = p == a ? hs : hs + 3 * T;
    p->col_off.assign(c, c + T);
    p->nnz.assign(h, h + T);
    p->maxdeg.assign(h + T, h + 2 * T);
    p->nerows.assign(h + 2 * T, h + 3 * T);
  }
  return BBTC_OK;
}

// Layout kernels are grid-stride loops: no more blocks than the largest array
// needs (a tiny graph's layout leaves the GPU to others), at most the
// context's cap.
int layout_grid(const bbtc_ctx* ctx, uint32_t n, uint64_t m, uint32_t P) {
  const uint64_t span = std::max<uint64_t>(m, (uint64_t)P * ((uint64_t)n + P));
  return (int)std::min<uint64_t>((uint64_t)ctx->sms * ctx->layout_blocks_per_sm,
                                 std::max<uint64_t>(ctx->sms, (span + 2047) / 2048));
}

uint64_t block_bytes(const BlockTiles& t, bool rec) {
  return (t.rp_len + t.col_len + t.erow_len) * sizeof(uint32_t) + (rec ? t.col_len * sizeof(uint2) : 0);
}

}  // namespace

void BlockTiles::release(cudaStream_t s) {
  if (d_rp) cudaFreeAsync(d_rp, s);
  if (d_col) cudaFreeAsync(d_col, s);
  if (d_rec) cudaFreeAsync(d_rec, s);
  if (d_erow) cudaFreeAsync(d_erow, s);
  d_rp = d_col = d_erow = nullptr;
  d_rec = nullptr;
}

DevTile dev_tile(const BlockTiles& t, const std::vector<uint32_t>& cuts, uint32_t x, uint32_t y) {
  DevTile d{};
  const uint32_t id = x * t.P + y;
  d.H = cuts[x + 1] - cuts[x];
  d.W = cuts[y + 1] - cuts[y];
  d.nnz = t.nnz[id];
  d.maxdeg = t.maxdeg[id];
  if (d.nnz) {
    d.rp = t.d_rp + t.rp_off[id];
    d.col = t.d_col + t.col_off[id];
    d.rec = t.d_rec ? reinterpret_cast<const uint2*>(t.d_rec) + t.col_off[id] : nullptr;
    d.erow = t.d_erow + t.col_off[id] / 32 + id;
  } else {
    d.rp = d.col = d.erow = nullptr;
    d.rec = nullptr;
  }
  return d;
}

// Layout scratch a context keeps between builds: the temporaries of a graph
// of up to about five million edges (about 45 bytes per edge); a larger
// build allocates its own and frees them at its end.
constexpr size_t kScratchKeep = 256ull << 20;

// Makes the context's kept scratch the running build's for the scope's
// lifetime, then grows the kept block to what the build asked for (a quarter
// more, at most kScratchKeep).  The kept block is a cache: when growing it
// fails the next build allocates as before, so it bypasses the allocation
// fault hook.  Its old block is freed behind the build's work on the stream.
struct ScratchScope {
  bbtc_ctx* ctx;
  cudaStream_t s;
  Scratch arena;
  Scratch* prev;
  ScratchScope(bbtc_ctx* c, cudaStream_t st) : ctx(c), s(st), prev(t_scratch) {
    arena.base = c->d_scratch;
    arena.cap = c->scratch_cap;
    t_scratch = &arena;
  }
  ~ScratchScope() {
    t_scratch = prev;
    if (arena.want <= ctx->scratch_cap || arena.want > kScratchKeep) return;
    if (ctx->d_scratch) cudaFreeAsync(ctx->d_scratch, s);
    ctx->d_scratch = nullptr;
    ctx->scratch_cap = 0;
    const size_t cap = std::min(kScratchKeep, ((arena.want + arena.want / 4) + (1u << 20) - 1) & ~size_t((1u << 20) - 1));
    void* p = nullptr;
    if (cudaMallocAsync(&p, cap, s) == cudaSuccess) {
      ctx->d_scratch = static_cast<char*>(p);
      ctx->scratch_cap = cap;
    } else {
      cudaGetLastError();
    }
  }
  ScratchScope(const ScratchScope&) = delete;
  ScratchScope& operator=(const ScratchScope&) = delete;
};

int build_layout(bbtc_graph* g, const uint32_t* in_indptr, const uint32_t* in_indices, bool host) {
  Range range("bbtc upload + layout");
  bbtc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  ScratchScope scratch(ctx, s);
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const uint32_t P = g->P;
  const uint32_t T = P * P;
  const int grid = layout_grid(ctx, n, m, P);
  cudaEvent_t ev0, ev1;
  BBTC_CUDA(cudaEventCreate(&ev0));
  BBTC_CUDA(cudaEventCreate(&ev1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } evg{ev0, ev1};
  BBTC_CUDA(cudaEventRecord(ev0, s));

  // the graph keeps its own copy of the oriented CSR: the fused task rows probe it
  {
    cudaError_t e1 = dev_malloc(&g->d_indptr, ((size_t)n + 1) * sizeof(uint32_t), s);
    cudaError_t e2 = dev_malloc(&g->d_indices, std::max<uint64_t>(m, 1) * sizeof(uint32_t) + 16, s);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
      cudaGetLastError();
      return fail(BBTC_ERR_NOMEM, "device allocation of the CSR copy failed");
    }
    const cudaMemcpyKind kind = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    // host copies in 8 MiB pieces: a copy engine runs one copy at a time, and
    // another stream's small upload then waits behind one piece, not behind
    // a whole large graph (273 MB at R-MAT s22: about 5 ms)
    // With an upload window (the server's large requests) at most that many
    // pieces are queued at once, so the copy engines' queues never hold a
    // large graph's whole upload ahead of another stream's small one.
    const uint32_t window = host ? ctx->upload_window : 0;
    cudaEvent_t evs[8] = {};
    struct EvRing {
      cudaEvent_t* e;
      ~EvRing() {
        for (int i = 0; i < 8; i++)
          if (e[i]) cudaEventDestroy(e[i]);
      }
    } ring{evs};
    uint32_t issued = 0;
    uint32_t by_kernel = 0;
    auto mapped = [&](const void* src, size_t bytes) {
      return host && bytes <= ctx->zero_copy_bytes && mapped_host_range(src, bytes);
    };
    // arrays that the SMs read over the host link, copied by one kernel launch
    uint32_t* kdst[2] = {nullptr, nullptr};
    const uint32_t* ksrc[2] = {nullptr, nullptr};
    uint64_t kwords[2] = {0, 0};
    auto copy = [&](void* dst, const void* src, size_t bytes) -> int {
      if (mapped(src, bytes)) {
        kdst[by_kernel] = static_cast<uint32_t*>(dst);
        ksrc[by_kernel] = static_cast<const uint32_t*>(src);
        kwords[by_kernel] = bytes / 4;
        by_kernel++;
        return BBTC_OK;
      }
      const size_t piece = host ? (size_t)8 << 20 : bytes;
      for (size_t o = 0; o < bytes; o += piece) {
        if (window) {
          cudaEvent_t& ev = evs[issued % std::min<uint32_t>(window, 8)];
          if (ev) BBTC_CUDA(cudaEventSynchronize(ev));
          else BBTC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        }
        BBTC_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o,
                                  std::min(piece, bytes - o), kind, s));
        if (window) BBTC_CUDA(cudaEventRecord(evs[issued % std::min<uint32_t>(window, 8)], s));
        issued++;
      }
      return BBTC_OK;
    };
    BBTC_TRY(copy(g->d_indptr, in_indptr, ((size_t)n + 1) * sizeof(uint32_t)));
    if (m) BBTC_TRY(copy(g->d_indices, in_indices, m * sizeof(uint32_t)));
    if (by_kernel) {
      const uint64_t words = std::max(kwords[0], kwords[1]);
      const uint64_t blocks = std::max<uint64_t>(1, (words + 4095) / 4096);
      BBTC_TRY(launch_layout(ctx, k_copy_mapped, (int)std::min<uint64_t>(blocks, 2ull * ctx->sms), 256, s, kdst[0],
                             ksrc[0], kwords[0], kdst[1], ksrc[1], kwords[1]));
    }
    g->zero_copy = by_kernel > 0;
  }
  const uint32_t* d_indptr = g->d_indptr;
  const uint32_t* d_indices = g->d_indices;

  DevBuf d_cuts, rows, stats_r, coloff_r, wflags, wpos, eids_in;
  BBTC_TRY(dalloc(wflags, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(wpos, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(d_cuts, (g->cuts.size() + 1) * sizeof(uint32_t), s));  // the cuts, then the contract flags
  BBTC_TRY(dalloc(rows, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(stats_r, 4 * T * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(coloff_r, T * sizeof(uint64_t), s));
  BBTC_TRY(dalloc(eids_in, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
  uint32_t* d_bad = d_cuts.as<uint32_t>() + g->cuts.size();
  {
    // one copy: the cut vector and a zero flags word
    uint32_t* h = reinterpret_cast<uint32_t*>(ctx->h_stage + kStageCuts);
    std::memcpy(h, g->cuts.data(), g->cuts.size() * sizeof(uint32_t));
    h[g->cuts.size()] = 0;
    BBTC_CUDA(cudaMemcpyAsync(d_cuts.p, h, (g->cuts.size() + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  }
  // The contract check runs first; its flags are read back with the tile
  // statistics at the end, and every kernel between that indexes by the input
  // returns at once when they are set, so no host round trip splits the build.
  if (n > 0) {
    BBTC_TRY(launch_layout(ctx, k_expand_check, grid, 256, s, d_indptr, d_indices, n, m, rows.as<uint32_t>(), d_bad,
                           wflags.as<uint32_t>(), eids_in.as<uint32_t>()));
  } else if (m > 0) {
    BBTC_CUDA(cudaMemsetAsync(d_bad, 0xff, sizeof(uint32_t), s));  // edges without rows
  }

  // the forward block CSR waits until something needs it (ensure_fwd): the
  // fused task rows read only the reversed one

  // word-compressed rows (the fused task rows stream these); k_expand_check wrote the flags
  {
    cudaError_t e1 = dev_malloc(&g->d_words, std::max<uint64_t>(m, 1) * sizeof(uint2) + 16, s);
    cudaError_t e2 = dev_malloc(&g->d_wptr, ((size_t)n + 1) * sizeof(uint32_t), s);
    cudaError_t e3 = dev_malloc(&g->d_desc, ((size_t)n + 1) * sizeof(uint4), s);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
      cudaGetLastError();
      return fail(BBTC_ERR_NOMEM, "device allocation of the word-compressed rows failed");
    }
    if (m > 0) {
      size_t tb = 0;
      BBTC_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, wflags.as<uint32_t>(), wpos.as<uint32_t>(), (int64_t)m, s));
      DevBuf tmp;
      BBTC_TRY(dalloc(tmp, tb, s));
      BBTC_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tb, wflags.as<uint32_t>(), wpos.as<uint32_t>(), (int64_t)m, s));
      BBTC_TRY(launch_layout(ctx, k_word_fill, grid, 256, s, d_indices, wflags.as<uint32_t>(), wpos.as<uint32_t>(), m,
                             reinterpret_cast<uint2*>(g->d_words), d_bad));
    } else {
      BBTC_CUDA(cudaMemsetAsync(g->d_words, 0, sizeof(uint2) + 16, s));
    }
    BBTC_TRY(launch_layout(ctx, k_word_rowptr, grid, 256, s, d_indptr, d_indices, wpos.as<uint32_t>(), n, m,
                           g->d_wptr, static_cast<uint4*>(g->d_desc), d_bad));
  }

  // reversed graph: a stable sort of (column, forward edge id) by column keeps
  // every in-list ordered by source
  {
    DevBuf keys_out, eids_out, rev_indptr, rev_cols;
    BBTC_TRY(dalloc(keys_out, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
    BBTC_TRY(dalloc(eids_out, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
    BBTC_TRY(dalloc(rev_cols, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
    BBTC_TRY(dalloc(rev_indptr, ((size_t)n + 1) * sizeof(uint32_t), s));
    if (m > 0) {
      int end_bit = 1;
      while (end_bit < 32 && (1ull << end_bit) < (uint64_t)n) end_bit++;
      size_t tmp_bytes = 0;
      BBTC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_indices, keys_out.as<uint32_t>(),
                                                eids_in.as<uint32_t>(), eids_out.as<uint32_t>(), (int64_t)m, 0,
                                                end_bit, s));
      DevBuf tmp;
      BBTC_TRY(dalloc(tmp, tmp_bytes, s));
      BBTC_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, d_indices, keys_out.as<uint32_t>(),
                                                eids_in.as<uint32_t>(), eids_out.as<uint32_t>(), (int64_t)m, 0,
                                                end_bit, s));
    }
    if (m > 0) {
      BBTC_TRY(launch_layout(ctx, k_gather, grid, 256, s, rows.as<uint32_t>(), eids_out.as<uint32_t>(), m,
                             rev_cols.as<uint32_t>(), d_bad));
    }
    BBTC_TRY(launch_layout(ctx, k_rev_indptr, grid, 256, s, keys_out.as<uint32_t>(), m, n, rev_indptr.as<uint32_t>(),
                           d_bad));
    // reversed entries: row = column vertex v (keys), column = source u, record of forward edge (u, v)
    BBTC_TRY(build_block(ctx, g->rev, rev_indptr.as<uint32_t>(), rev_cols.as<uint32_t>(), keys_out.as<uint32_t>(),
                         n, m, g->cuts, d_cuts.as<uint32_t>(), eids_out.as<uint32_t>(), wpos.as<uint32_t>(),
                         g->d_wptr, d_indptr, d_indices, reinterpret_cast<const uint2*>(g->d_words),
                         stats_r.as<uint32_t>(), coloff_r.as<uint64_t>(), d_bad, grid));
  }
  // the host needs the tile statistics and the contract flags only now: one read-back
  uint32_t hbad = 0;
  BBTC_TRY(fetch_stats(ctx, nullptr, g->rev, nullptr, nullptr, stats_r.as<uint32_t>(), coloff_r.as<uint64_t>(), s,
                       d_bad, &hbad));
  if (hbad) {
    std::string why;
    if (hbad == 0xffffffffu) why += " edges but no rows;";
    else {
      if (hbad & 1) why += " indptr[0] != 0;";
      if (hbad & 2) why += " indptr[n] != m;";
      if (hbad & 4) why += " row pointers decrease or exceed m;";
      if (hbad & 8) why += " a column id >= n;";
      if (hbad & 16) why += " a row is not strictly increasing (unsorted or duplicate ids);";
    }
    return fail(BBTC_ERR_INPUT, "CSR breaks the input contract:" + why);
  }
  BBTC_CUDA(cudaEventRecord(ev1, s));
  BBTC_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  BBTC_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  g->layout_ms = ms;
  g->device_bytes = block_bytes(g->rev, true) + ((uint64_t)n + 1 + m) * sizeof(uint32_t) + 64 * sizeof(uint64_t) +
                    m * sizeof(uint2) + ((uint64_t)n + 1) * (sizeof(uint32_t) + sizeof(uint4));
  return BBTC_OK;
}

namespace {

int build_fwd(bbtc_graph* g) {
  Range range("bbtc forward tiles");
  bbtc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  BBTC_CUDA(cudaSetDevice(ctx->device));
  const uint32_t n = g->n, P = g->P, T = P * P;
  const uint64_t m = g->m;
  const int grid = layout_grid(ctx, n, m, P);
  DevBuf d_cuts, bad, rows, stats, coloff;
  BBTC_TRY(dalloc(d_cuts, g->cuts.size() * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(bad, sizeof(uint32_t), s));
  BBTC_TRY(dalloc(rows, std::max<uint64_t>(m, 1) * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(stats, 4 * T * sizeof(uint32_t), s));
  BBTC_TRY(dalloc(coloff, T * sizeof(uint64_t), s));
  {
    uint32_t* h = reinterpret_cast<uint32_t*>(ctx->h_stage + kStageCuts);
    std::memcpy(h, g->cuts.data(), g->cuts.size() * sizeof(uint32_t));
    BBTC_CUDA(cudaMemcpyAsync(d_cuts.p, h, g->cuts.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  }
  BBTC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(uint32_t), s));
  if (n > 0) {
    // row id of every edge (the CSR passed validation when it was uploaded)
    BBTC_TRY(launch_layout(ctx, k_expand_check, grid, 256, s, g->d_indptr, g->d_indices, n, m, rows.as<uint32_t>(),
                           bad.as<uint32_t>(), nullptr, nullptr));
  }
  BBTC_TRY(build_block(ctx, g->fwd, g->d_indptr, g->d_indices, rows.as<uint32_t>(), n, m, g->cuts,
                       d_cuts.as<uint32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                       stats.as<uint32_t>(), coloff.as<uint64_t>(), bad.as<uint32_t>(), grid));
  BBTC_TRY(fetch_stats(ctx, nullptr, g->fwd, nullptr, nullptr, stats.as<uint32_t>(), coloff.as<uint64_t>(), s));
  g->fwd_built = true;
  g->device_bytes += block_bytes(g->fwd, false);
  return BBTC_OK;
}

}  // namespace

int ensure_fwd(bbtc_graph* g) {
  if (g->fwd_built) return BBTC_OK;
  const int rc = build_fwd(g);
  if (rc != BBTC_OK) {
    // a failed build (say, out of memory half way) leaves nothing behind: the
    // frees are stream-ordered after whatever of it was enqueued
    g->fwd.release(g->ctx->stream);
    g->fwd = BlockTiles();
  }
  return rc;
}

}  // namespace bbtc

// Read the whole layout back and check it on the host (debug aid: it copies
// every array, so it costs about the graph's device bytes in host memory and
// PCIe time).  The forward block CSR is checked when it has been built.
int bbtc_graph_validate(const bbtc_graph* g) {
  using namespace bbtc;
  static_assert(check::kNoSeg == kNoSegment, "empty-tile marker");
  if (!g) return fail(BBTC_ERR_ARG, "NULL graph");
  bbtc_ctx* ctx = g->ctx;
  Range range("bbtc validate");
  cudaStream_t s = ctx->stream;
  BBTC_CUDA(cudaSetDevice(ctx->device));
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const uint64_t mm = std::max<uint64_t>(m, 1);
  auto get = [&](std::vector<uint32_t>& h, const void* d, uint64_t words) -> int {
    h.assign(words, 0);
    if (words) BBTC_CUDA(cudaMemcpyAsync(h.data(), d, words * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    return BBTC_OK;
  };
  std::vector<uint32_t> indptr, indices, wptr, pairs, desc;
  BBTC_TRY(get(desc, g->d_desc, 4 * ((uint64_t)n + 1)));
  BBTC_TRY(get(indptr, g->d_indptr, (uint64_t)n + 1));
  BBTC_TRY(get(indices, g->d_indices, mm));
  BBTC_TRY(get(wptr, g->d_wptr, (uint64_t)n + 1));
  BBTC_TRY(get(pairs, g->d_words, 2 * mm));
  BBTC_CUDA(cudaStreamSynchronize(s));
  check::Csr c{n, m, indptr.data(), indices.data()};
  check::Words w{wptr.data(), pairs.data(), mm};
  std::string why = check::csr(c);
  if (why.empty()) why = check::words(c, w);
  if (why.empty()) why = check::descs(c, w, desc.data());
  std::vector<uint32_t> tp, tc;
  if (why.empty()) check::transpose(c, tp, tc);
  const check::Csr tr{n, m, tp.data(), tc.data()};
  for (int pass = 0; pass < 2 && why.empty(); pass++) {
    const BlockTiles& bt = pass == 0 ? g->rev : g->fwd;
    if (pass == 1 && !g->fwd_built) break;
    std::vector<uint32_t> rp, col, erow, rec;
    BBTC_TRY(get(rp, bt.d_rp, bt.rp_len));
    BBTC_TRY(get(col, bt.d_col, bt.col_len));
    BBTC_TRY(get(erow, bt.d_erow, bt.erow_len));
    if (bt.d_rec) BBTC_TRY(get(rec, bt.d_rec, 2 * bt.col_len));
    BBTC_CUDA(cudaStreamSynchronize(s));
    check::Tiles t;
    t.P = g->P;
    t.cuts = g->cuts.data();
    t.rp_off = bt.rp_off.data();
    t.col_off = bt.col_off.data();
    t.nnz = bt.nnz.data();
    t.maxdeg = bt.maxdeg.data();
    t.nerows = bt.nerows.data();
    t.rp = rp.data();
    t.rp_len = bt.rp_len;
    t.col = col.data();
    t.col_len = bt.col_len;
    t.erow = erow.data();
    t.erow_len = bt.erow_len;
    t.rec = bt.d_rec ? rec.data() : nullptr;
    if (pass == 0 && !t.rec) why = "reversed tiles: no forward-edge records";
    else why = check::tiles(pass == 0 ? "reversed tiles" : "forward tiles", pass == 0 ? tr : c, t, w);
  }
  if (!why.empty()) return fail(BBTC_ERR_LAYOUT, "device layout check failed: " + why);
  return BBTC_OK;
}

// Intersection kernels, the device work queue and the launch paths.
//
// A task (i, j, k) contributes sum_{r in part i} sum_{b in ab[r]} |ac[r] ∩ bc[b]|
// (the reference's SparseKernel / DenseKernel, src/triangle_counting/
// gpu_sparse_kernel.cu:6-49 and gpu_dense_kernel.cu:3-47, one thread per row
// of ab).  Here the sum is taken one *pivot row* at a time: the pivot row
// becomes a membership structure in the warp's shared memory and the rows it
// meets are streamed against it.
//
// Per-task execution (plain form, explicit task lists):
//   v-centric (default): pivot = row b of bc (vertex v of part j); the rows
//     streamed are ac[u] for every u with b in ab[u] -- column b of ab, read
//     from the reversed tile (j, i).  With the degree order the ac rows are the
//     shorter side, so this probes sum d_k(u) ids where the reference's bitmap
//     form probes sum d_k(v).
//   u-centric (the reference's row order, BBTC_KERNEL_MERGE): pivot = ac[r],
//     the rows bc[b] for b in ab[r] are streamed against it.
//
// Fused task rows (persistent form over the whole task list): the tasks
// (i, j, k) for all k >= j share their ab tile, and their sum over k is
// sum_{(u, v) in ab} |N+(u) ∩ N+(v) ∩ [cuts[j], ∞)|.  One pass over the
// reversed tile (j, i) takes it: per pivot v the row N+(v) from cuts[j] on
// (for a CSR oriented from lower to higher ids, the whole row) is the
// structure, and per in-edge (u, v) the ids of N+(u) that can meet it are
// streamed -- their range is stored with the in-edge, so no row pointer is
// chased.  This visits each edge once instead of once per k.
//
// Membership structures: a bitmap (of the column part, or of the pivot row's
// id span), a sorted copy searched by bisection, or -- for pivot rows longer
// than the shared buffer -- bisection in global memory.
//
// Work units are runs of `unit_edges` consecutive entries of the rows tile.
// In the persistent form every warp of a grid sized to the SM count claims
// units from one atomic head over all tasks (cost-sorted, heaviest first); in
// the plain form each task is one launch whose warps stride over its units.
// Inside a unit the rows met by 32 entries are concatenated and walked 32
// consecutive ids at a time (see probe_entries).
#include <algorithm>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <sstream>

#include "internal.h"

namespace bbtc {

namespace {

constexpr uint32_t FULL = 0xffffffffu;
// per warp after its bitmap: 33 segment starts, 32 bases, a pad word and the
// 8-byte aligned FusedFrame (28 words), rounded up to an even count
constexpr uint32_t kSegWords = 96;
constexpr uint32_t kFrameOffset = 66;  // words after the bitmap
// per-warp bulk-staging state of the per-task kernels, after the bitmap:
// an mbarrier (8 bytes) at kBarOffset, its phase bit and a "staging off" flag
constexpr uint32_t kBarOffset = 92;
constexpr uint32_t kPhaseOffset = 94;
constexpr uint32_t kStageOffFlag = 95;
constexpr uint32_t kStageMin = 64;         // pivot rows this long or longer are staged by one bulk copy
constexpr uint32_t kWaitLimit = 1u << 20;  // try_wait polls before a staging copy is given up
// values of the warp's staging flag (state[kStageOffFlag])
constexpr uint32_t kStageOn = 0, kStageOff = 1, kStageDead = 2;
constexpr uint32_t kSplitList = 128; // split pivots: room for the ids below the bitmap window

// ---- bulk copies into shared memory (cp.async.bulk + mbarrier) ------------

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One lane: copy `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global to shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_to_shared(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier plain stores to dst come first
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Wait for the phase with parity `parity` of `bar` to complete; false when
// it has not after `limit` polls.  Warp-uniform: true only when every lane
// saw the phase complete (each lane's own wait orders its later reads).
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
  bool done_all = false;
  for (uint32_t i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) {
      done_all = true;
      break;
    }
  }
  return __all_sync(FULL, done_all);
}

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t n, uint32_t x) {
  uint32_t lo = 0;
  while (n > 0) {
    const uint32_t half = n >> 1;
    if (a[lo + half] < x) {
      lo += half + 1;
      n -= half + 1;
    } else {
      n = half;
    }
  }
  return lo;
}

struct PivotView {
  const uint32_t* row;  // global pivot row
  uint32_t len;
  uint32_t base;  // bitmap bit 0 <-> id `base`
  uint32_t cap;   // a bit of the warp's last buffer word, which stays zero
  uint32_t first, last;
  const uint32_t* res;  // split kind: the pivot ids below `base`, sorted
  uint32_t rlen;
};

// First p in [from, n) with a[p] >= x (n if none) for a sorted a, given
// a[from - 1] < x: steps of 1, 2, 4, ... from `from`, then bisection of the
// last step.  A lane probing increasing ids of one row against a long pivot
// row moves forward from its previous position instead of bisecting the
// whole row again (skewed degrees: long pivot rows, short probe rows).
__device__ __forceinline__ uint32_t gallop_lb(const uint32_t* __restrict__ a, uint32_t n, uint32_t from, uint32_t x) {
  if (from >= n || a[from] >= x) return from;
  uint32_t lo = from, step = 1;  // a[lo] < x
  while (lo + step < n && a[lo + step] < x) {
    lo += step;
    step <<= 1;
  }
  uint32_t L = lo + 1;
  uint32_t len = min(lo + step, n) - L;  // the answer is in [L, L + len]
  while (len > 0) {
    const uint32_t half = len >> 1;
    if (a[L + half] < x) {
      L += half + 1;
      len -= half + 1;
    } else {
      len = half;
    }
  }
  return L;
}

template <uint32_t KIND>
__device__ __forceinline__ uint32_t member(const uint32_t* bm, const PivotView& pv, uint32_t x) {
  if constexpr (KIND == kPivotBitmap) {
    // ids outside the pivot's span (below base they wrap high) land on the
    // always-zero last word: no branch
    const uint32_t y = min(x - pv.base, pv.cap);
    return (bm[y >> 5] >> (y & 31)) & 1u;
  } else if constexpr (KIND == kPivotSplit) {
    if (x >= pv.base) {
      const uint32_t y = min(x - pv.base, pv.cap);
      return (bm[y >> 5] >> (y & 31)) & 1u;
    }
    if (x < pv.first) return 0;
    const uint32_t p = lower_bound_u32(pv.res, pv.rlen, x);
    return (p < pv.rlen && pv.res[p] == x) ? 1u : 0u;
  } else if constexpr (KIND == kPivotList) {
    if (x < pv.first || x > pv.last) return 0;
    const uint32_t p = lower_bound_u32(bm, pv.len, x);
    return (p < pv.len && bm[p] == x) ? 1u : 0u;
  } else {
    if (x < pv.first || x > pv.last) return 0;
    const uint32_t p = lower_bound_u32(pv.row, pv.len, x);
    return (p < pv.len && pv.row[p] == x) ? 1u : 0u;
  }
}

// Hits of one word-compressed pair (32-id word w.x, bit mask w.y).  The
// bitmap kinds use a word-aligned base, so a pair meets one bitmap word; ids
// below a split pivot's window, and the list kinds, test the set bits one by one.
template <uint32_t KIND>
__device__ __forceinline__ uint32_t member_word(const uint32_t* bm, const PivotView& pv, uint2 w) {
  if constexpr (KIND == kPivotBitmap) {
    const uint32_t yw = min(w.x - (pv.base >> 5), pv.cap >> 5);
    return __popc(w.y & bm[yw]);
  } else if constexpr (KIND == kPivotRank) {
    // pv.base: the pivot's first word; pv.cap: its span in words; bm: one
    // (presence bits, index of the block's first pair) entry per 32 words;
    // pv.res: the pivot's masks in pair order.  A word the pivot lacks costs
    // one 8-byte load.
    const uint32_t rel = w.x - pv.base;  // words below the first wrap high
    if (rel >= pv.cap) return 0;
    const uint2 e = reinterpret_cast<const uint2*>(bm)[rel >> 5];
    const uint32_t bit = 1u << (rel & 31);
    if (!(e.x & bit)) return 0;
    return __popc(w.y & pv.res[e.y + __popc(e.x & (bit - 1u))]);
  } else {
    if constexpr (KIND == kPivotSplit) {
      if (w.x >= (pv.base >> 5)) return __popc(w.y & bm[min(w.x - (pv.base >> 5), pv.cap >> 5)]);
    }
    uint32_t hits = 0;
    uint32_t mask = w.y;
    while (mask) {
      const uint32_t x = (w.x << 5) | (uint32_t)(__ffs(mask) - 1);
      mask &= mask - 1;
      hits += member<KIND>(bm, pv, x);
    }
    return hits;
  }
}

// Segment of the probe ids met by entry q of the rows tile.
struct TileSegs {  // per task: the probe tile's row r = rows.col[q]
  const uint32_t* __restrict__ rcol;
  const uint32_t* __restrict__ rp;
  __device__ __forceinline__ void get(uint32_t q, uint32_t& start, uint32_t& len) const {
    const uint32_t r = rcol[q];
    start = rp[r];
    len = rp[r + 1] - start;
  }
};
struct RecSegs {  // fused: the stored (start, end) of N+(u) after v
  const uint2* __restrict__ rec;
  __device__ __forceinline__ void get(uint32_t q, uint32_t& start, uint32_t& len) const {
    const uint2 r = rec[q];
    start = r.x;
    len = r.y - r.x;
  }
};

// Probe the rows met by entries [e, ee) against the pivot structure; returns
// this lane's hit count.
//
// The rows met by a batch of 32 entries are concatenated and walked 32 ids at
// a time, lane l taking ids l, l + 32, l + 64, ..., so each warp load reads
// consecutive ids.  Every lane keeps a pointer to the row that owns its
// current id (found once per batch by bisection of the 33 row starts in
// shared memory) and moves it forward when its id passes the row's end --
// less than once per window on average -- so the owner costs one compare per
// id.  Four windows are loaded before any is tested.
template <uint32_t KIND, bool WORDS, class Segs>
__device__ __forceinline__ uint32_t probe_entries(const Segs& segs, uint32_t e, uint32_t ee,
                                                  const uint32_t* __restrict__ prb_col, const uint32_t* bm,
                                                  uint32_t* sstart, uint32_t* sbase, const PivotView& pv,
                                                  uint32_t lane) {
  uint32_t hits = 0;
  for (uint32_t base = e; base < ee; base += 32) {
    const uint32_t q = base + lane;
    uint32_t start = 0, len = 0;
    if (q < ee) segs.get(q, start, len);
    uint32_t incl = len;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, incl, d);
      if (lane >= d) incl += t;
    }
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    if (total == 0) continue;
    const uint32_t excl = incl - len;
    sstart[lane] = excl;
    sbase[lane] = start - excl;  // modular: sbase + id is the id's position for ids of this row
    if (lane == 31) sstart[32] = total;
    __syncwarp();
    // owner of id = lane: the last row whose start is <= lane (empty rows share starts)
    uint32_t owner = 0;
#pragma unroll
    for (uint32_t step = 16; step > 0; step >>= 1)
      if (sstart[owner + step] <= lane) owner += step;
    uint32_t nb = sstart[owner + 1];
    uint32_t bs = sbase[owner];
    uint32_t gown = 0xffffffffu, gpos = 0;  // global kind: probe row and position of the last search
    for (uint32_t c = 0; c < total; c += 128) {
      if constexpr (WORDS) {
        const uint2* __restrict__ words = reinterpret_cast<const uint2*>(prb_col);
        uint2 x[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t id = c + 32u * k + lane;
          ok[k] = id < total;
          x[k] = make_uint2(0, 0);
          if (ok[k]) {
            while (id >= nb) {
              owner++;
              nb = sstart[owner + 1];
              bs = sbase[owner];
            }
            x[k] = __ldg(words + bs + id);
          }
        }
#pragma unroll
        for (int k = 0; k < 4; k++) hits += ok[k] ? member_word<KIND>(bm, pv, x[k]) : 0u;
      } else {
        uint32_t x[4];
        bool ok[4];
        uint32_t own[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t id = c + 32u * k + lane;
          ok[k] = id < total;
          x[k] = 0;
          if (ok[k]) {
            while (id >= nb) {
              owner++;
              nb = sstart[owner + 1];
              bs = sbase[owner];
            }
            x[k] = __ldg(prb_col + bs + id);
          }
          own[k] = owner;
        }
        if constexpr (KIND == kPivotGlobal) {
          // galloping search in the pivot row from this lane's last position
          // in the same probe row (ids of one row come in increasing order)
#pragma unroll
          for (int k = 0; k < 4; k++) {
            if (!ok[k]) continue;
            if (own[k] != gown) {
              gown = own[k];
              gpos = 0;
            }
            if (x[k] < pv.first || x[k] > pv.last) continue;
            gpos = gallop_lb(pv.row, pv.len, gpos, x[k]);
            hits += (gpos < pv.len && pv.row[gpos] == x[k]) ? 1u : 0u;
          }
        } else {
#pragma unroll
          for (int k = 0; k < 4; k++) hits += ok[k] ? member<KIND>(bm, pv, x[k]) : 0u;
        }
      }
    }
    __syncwarp();
  }
  return hits;
}

// Build the pivot structure, probe entries [e, ee), restore the buffer to zero.
// Split kind: ids >= base go to a bitmap of `words` words, the first `rlen`
// ids of the row (those below base) to a sorted list after the zero word.
template <uint32_t KIND, bool WORDS, class Segs>
__device__ __forceinline__ uint32_t pivot_pass(const uint32_t* __restrict__ prow, uint32_t pd, uint32_t base,
                                               uint32_t words, uint32_t rlen, const Segs& segs, uint32_t e,
                                               uint32_t ee, const uint32_t* __restrict__ prb_col, uint32_t* bm,
                                               uint32_t* sstart, uint32_t* sbase, uint32_t lane) {
  uint32_t* res = bm + words + 1;
  if constexpr (KIND == kPivotBitmap) {
    for (uint32_t i = lane; i < pd; i += 32) {
      const uint32_t y = prow[i] - base;
      atomicOr(&bm[y >> 5], 1u << (y & 31));
    }
  } else if constexpr (KIND == kPivotSplit) {
    for (uint32_t i = lane; i < pd; i += 32) {
      const uint32_t x = prow[i];
      if (i < rlen) {
        res[i] = x;
      } else {
        const uint32_t y = x - base;
        atomicOr(&bm[y >> 5], 1u << (y & 31));
      }
    }
  } else if constexpr (KIND == kPivotList) {
    for (uint32_t i = lane; i < pd; i += 32) bm[i] = prow[i];
  }
  __syncwarp();
  PivotView pv;
  pv.row = prow;
  pv.len = pd;
  pv.base = base;
  pv.cap = words * 32;  // callers keep words < the buffer size, so word `words` is never set
  pv.first = prow[0];
  pv.last = prow[pd - 1];
  pv.res = res;
  pv.rlen = rlen;
  const uint32_t hits = probe_entries<KIND, WORDS>(segs, e, ee, prb_col, bm, sstart, sbase, pv, lane);
  // the buffer is all-zero between pivots whatever kind used it last: the
  // persistent queue hands one warp bitmap and list work in any order
  __syncwarp();
  if constexpr (KIND == kPivotBitmap) {
    if (pd < words) {
      for (uint32_t i = lane; i < pd; i += 32) bm[(prow[i] - base) >> 5] = 0;
    } else {
      for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
    }
  } else if constexpr (KIND == kPivotSplit) {
    if (pd - rlen < words) {
      for (uint32_t i = lane + rlen; i < pd; i += 32) bm[(prow[i] - base) >> 5] = 0;
    } else {
      for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
    }
    for (uint32_t i = lane; i < rlen; i += 32) res[i] = 0;
  } else if constexpr (KIND == kPivotList) {
    for (uint32_t i = lane; i < pd; i += 32) bm[i] = 0;
  }
  __syncwarp();
  return hits;
}

// Row b of a tile holding entry e: the largest b with rp[b] <= e.
__device__ __forceinline__ uint32_t row_of(const uint32_t* __restrict__ rp, uint32_t H, uint32_t e) {
  uint32_t lo = 0, hi = H;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (rp[mid] <= e) lo = mid; else hi = mid;
  }
  return lo;
}

// Next row after b with an entry at or after e (a warp-wide scan of row ends).
__device__ __forceinline__ uint32_t next_row(const uint32_t* __restrict__ rp, uint32_t H, uint32_t b, uint32_t e,
                                             uint32_t lane) {
  b++;
  while (true) {
    const uint32_t idx = b + lane;
    const uint32_t v = idx < H ? rp[idx + 1] : 0xffffffffu;
    const uint32_t mask = __ballot_sync(FULL, v > e);
    if (mask) return b + __ffs(mask) - 1;
    b += 32;
  }
}

// One per-task work unit: entries [unit*K, min((unit+1)*K, nnz)) of the rows tile.
// Per-task pivot of the bitmap or list kind, staged in shared memory by one
// bulk copy (cp.async.bulk, the TMA engine; completion on the warp's
// mbarrier) of the 16-byte aligned span of the pivot row's column ids: the
// bitmap is then set, and cleared afterwards, from shared memory, and the
// list kind searches the staged span in place.  Returns false, having done
// nothing, when the row is short, the span does not fit the room left in the
// warp's buffer, or staging is off on this warp; the caller then loads the
// row itself (pivot_pass).  The column segment of a tile starts on a 16-byte
// boundary and the pool ends with a 16-byte tail, so the rounded span stays
// inside the allocation.
//
// A copy that has not landed after the wait limit voids the count (the
// error word; the host fails the call with BBTC_ERR_TIMEOUT).  The warp then
// waits once more, bounded, for the copy still in flight: if it lands, the
// staged span is cleared and the warp goes on without staging; if not, the
// warp may not touch its buffer again and stops (kStageDead), taking no more
// work.  `dbg` > 0 is the test hook of bbtc_debug_stage_timeout: no copy is
// issued, so the wait gives up after `dbg` polls with nothing in flight.
template <uint32_t KIND>
__device__ __forceinline__ bool staged_pass(const uint32_t* __restrict__ tile_col, uint32_t ps, uint32_t pd,
                                            uint32_t words, const TileSegs& segs, uint32_t e, uint32_t ee,
                                            const uint32_t* __restrict__ prb_col, uint32_t* bm, uint32_t bm_words,
                                            uint32_t* sstart, uint32_t* sbase, uint32_t lane, uint32_t* err,
                                            uint32_t dbg, unsigned long long& acc) {
  uint32_t* state = bm + bm_words;
  if (pd < kStageMin || state[kStageOffFlag] != kStageOn) return false;
  const uint32_t a0 = ps & ~3u, off = ps & 3u;
  const uint32_t span = ((ps + pd + 3u) & ~3u) - a0;  // words, a multiple of 4
  // bitmap kind: after the bitmap and its always-zero word; list kind: the list itself
  uint32_t* stage = KIND == kPivotList ? bm : bm + ((words + 1u + 3u) & ~3u);
  if (span > bm_words - (uint32_t)(stage - bm)) return false;
  uint64_t* bar = reinterpret_cast<uint64_t*>(state + kBarOffset);
  const uint32_t phase = state[kPhaseOffset];
  const uint32_t limit = dbg ? dbg : kWaitLimit;
  if (lane == 0 && !dbg) bulk_to_shared(stage, tile_col + a0, span * 4u, bar);
  const bool ok = bar_wait(bar, phase, limit);
  __syncwarp();
  if (!ok) {
    // the copy did not land in time: the count is void
    if (lane == 0) atomicOr(err, 1u);
    const bool landed = bar_wait(bar, phase, limit);  // drain the copy still in flight
    if (landed) {
      for (uint32_t i = lane; i < span; i += 32) stage[i] = 0;
      if (lane == 0) {
        state[kPhaseOffset] = phase ^ 1u;
        state[kStageOffFlag] = kStageOff;
      }
    } else if (lane == 0) {
      state[kStageOffFlag] = kStageDead;
    }
    __syncwarp();
    return true;
  }
  if (lane == 0) state[kPhaseOffset] = phase ^ 1u;
  const uint32_t* ids = stage + off;
  if constexpr (KIND == kPivotBitmap) {
    for (uint32_t i = lane; i < pd; i += 32) {
      const uint32_t y = ids[i];
      atomicOr(&bm[y >> 5], 1u << (y & 31));
    }
  }
  __syncwarp();
  PivotView pv;
  pv.row = tile_col + ps;
  pv.len = pd;
  pv.base = 0;
  pv.cap = words * 32;
  pv.first = ids[0];
  pv.last = ids[pd - 1];
  pv.res = nullptr;
  pv.rlen = 0;
  const uint32_t hits =
      probe_entries<KIND, false>(segs, e, ee, prb_col, KIND == kPivotList ? ids : bm, sstart, sbase, pv, lane);
  __syncwarp();
  // back to an all-zero buffer: the bitmap words the ids set, then the staged span
  if constexpr (KIND == kPivotBitmap) {
    if (pd < words) {
      for (uint32_t i = lane; i < pd; i += 32) bm[ids[i] >> 5] = 0;
    } else {
      for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
    }
    __syncwarp();
  }
  for (uint32_t i = lane; i < span; i += 32) stage[i] = 0;
  __syncwarp();
  acc += hits;
  return true;
}

// Set up a warp's staging state (kernel start, before any bulk copy).
__device__ __forceinline__ void staging_init(uint32_t* bm, uint32_t bm_words, uint32_t lane) {
  uint32_t* state = bm + bm_words;
  if (lane == 0) {
    bar_init(reinterpret_cast<uint64_t*>(state + kBarOffset));
    state[kPhaseOffset] = 0;
    state[kStageOffFlag] = kStageOn;
  }
  __syncwarp();
}

// True once a staging copy of this warp was given up while possibly still in
// flight: the warp stops working (its count is void already).
__device__ __forceinline__ bool staging_dead(const uint32_t* bm, uint32_t bm_words) {
  return bm[bm_words + kStageOffFlag] == kStageDead;
}

__device__ __noinline__ unsigned long long task_unit(const DevTask& tk, uint32_t unit, uint32_t* bm,
                                                     uint32_t* sstart, uint32_t* sbase, uint32_t lane,
                                                     uint32_t bm_words, uint32_t* err, uint32_t dbg) {
  const uint32_t* __restrict__ r_rp = tk.rows.rp;
  const uint32_t* __restrict__ p_rp = tk.pivot.rp;
  const uint32_t* __restrict__ p_col = tk.pivot.col;
  const TileSegs segs{tk.rows.col, tk.probe.rp};
  const uint32_t H = tk.rows.H;
  const uint64_t e0 = (uint64_t)unit * tk.unit_edges;
  const uint64_t e1w = e0 + tk.unit_edges;
  uint32_t e = (uint32_t)e0;
  const uint32_t e1 = e1w < tk.rows.nnz ? (uint32_t)e1w : tk.rows.nnz;
  uint32_t b = tk.rows.erow[e >> 5];  // units start at multiples of 32 entries
  unsigned long long acc = 0;
  while (e < e1) {
    const uint32_t ee = min(r_rp[b + 1], e1);
    const uint32_t ps = p_rp[b];
    const uint32_t pd = p_rp[b + 1] - ps;
    if (pd > 0) {
      const uint32_t* prow = p_col + ps;
      switch (tk.kind) {
        case kPivotBitmap:
          if (!staged_pass<kPivotBitmap>(p_col, ps, pd, tk.words, segs, e, ee, tk.probe.col, bm, bm_words, sstart,
                                         sbase, lane, err, dbg, acc))
            acc += pivot_pass<kPivotBitmap, false>(prow, pd, 0, tk.words, 0, segs, e, ee, tk.probe.col, bm, sstart,
                                                   sbase, lane);
          break;
        case kPivotList:
          if (!staged_pass<kPivotList>(p_col, ps, pd, 0, segs, e, ee, tk.probe.col, bm, bm_words, sstart, sbase, lane,
                                       err, dbg, acc))
            acc += pivot_pass<kPivotList, false>(prow, pd, 0, 0, 0, segs, e, ee, tk.probe.col, bm, sstart, sbase, lane);
          break;
        default:
          acc += pivot_pass<kPivotGlobal, false>(prow, pd, 0, 0, 0, segs, e, ee, tk.probe.col, bm, sstart, sbase, lane);
      }
      if (staging_dead(bm, bm_words)) return acc;
    }
    e = ee;
    if (e < e1) b = next_row(r_rp, H, b, e, lane);
  }
  return acc;
}

// The pivot of a fused task row (i, j): the tasks (i, j, k >= j) count the
// common neighbours w of an in-edge (u, v) with w in column parts k >= j,
// i.e. w >= lo = cuts[j] (the reference's tiles ac = (i, k), bc = (j, k),
// src/triangle_counting/gpu_sparse_kernel.cu:25-46).  Drops the ids of
// N+(v) below lo from the pivot row [ps, ps + pd) and from its word pairs
// [ws, ws + wn); mask0 clears the dropped ids that share the first kept
// pair's word.  Called only when N+(v) starts below lo, which a CSR oriented
// from lower to higher ids never does (every id of N+(v) exceeds v >= lo).
__device__ __noinline__ void pivot_suffix(const uint32_t* __restrict__ gi, const uint2* __restrict__ gw, uint32_t lo,
                                          uint32_t& ps, uint32_t& pd, uint32_t& ws, uint32_t& wn, uint32_t& mask0) {
  const uint32_t k = lower_bound_u32(gi + ps, pd, lo);
  ps += k;
  pd -= k;
  if (pd == 0) {
    wn = 0;
    return;
  }
  const uint32_t first = gi[ps];
  // first pair whose word holds `first` (a row's pair words strictly increase)
  uint32_t lo_p = 0, n = wn;
  while (n > 0) {
    const uint32_t half = n >> 1;
    if (gw[ws + lo_p + half].x < (first >> 5)) {
      lo_p += half + 1;
      n -= half + 1;
    } else {
      n = half;
    }
  }
  ws += lo_p;
  wn -= lo_p;
  mask0 = FULL << (first & 31);
}

// One fused task-row unit: in-edges [unit*K, ...) of the reversed tile (j, i).
__device__ __noinline__ unsigned long long fused_unit(const DevTask& tk, uint32_t unit, uint32_t* bm,
                                                      uint32_t* sstart, uint32_t* sbase, uint32_t lane,
                                                      uint32_t bm_words) {
  const uint32_t* __restrict__ r_rp = tk.rows.rp;
  const uint32_t* __restrict__ gp = tk.g_indptr;
  const uint32_t* __restrict__ gi = tk.g_indices;
  const RecSegs segs{tk.rows.rec};
  const uint32_t H = tk.rows.H;
  const uint64_t e0 = (uint64_t)unit * tk.unit_edges;
  const uint64_t e1w = e0 + tk.unit_edges;
  uint32_t e = (uint32_t)e0;
  const uint32_t e1 = e1w < tk.rows.nnz ? (uint32_t)e1w : tk.rows.nnz;
  uint32_t b = tk.rows.erow[e >> 5];  // units start at multiples of 32 entries
  unsigned long long acc = 0;
  while (e < e1) {
    const uint32_t ee = min(r_rp[b + 1], e1);
    const uint32_t v = tk.pivot_base + b;
    uint32_t ps = gp[v];
    uint32_t pd = gp[v + 1] - ps;
    if (pd > 0 && gi[ps] < tk.pivot_base) {
      // keep the ids in the task columns only (this pivot is built from ids)
      const uint32_t k = lower_bound_u32(gi + ps, pd, tk.pivot_base);
      ps += k;
      pd -= k;
    }
    if (pd > 0) {
      const uint32_t* prow = gi + ps;
      const uint32_t first = prow[0];
      const uint32_t last = prow[pd - 1];
      // word-aligned bitmap: a streamed pair meets exactly one bitmap word
      const uint32_t base = first & ~31u;
      const uint32_t span_words = (last >> 5) - (first >> 5) + 1;
      const uint32_t* gw = reinterpret_cast<const uint32_t*>(tk.g_words);
      if (span_words < bm_words) {
        acc += pivot_pass<kPivotBitmap, true>(prow, pd, base, span_words, 0, segs, e, ee, gw, bm, sstart, sbase,
                                              lane);
      } else {
        // bitmap over the top words of the row, the few ids below them in a short list
        const uint32_t wwords = bm_words - 1 - kSplitList;
        const uint32_t wbase = ((last >> 5) - (wwords - 1)) << 5;
        const uint32_t rlen = lower_bound_u32(prow, pd, wbase);
        if (rlen <= kSplitList)
          acc += pivot_pass<kPivotSplit, true>(prow, pd, wbase, wwords, rlen, segs, e, ee, gw, bm, sstart, sbase,
                                               lane);
        else if (pd <= bm_words)
          acc += pivot_pass<kPivotList, true>(prow, pd, 0, 0, 0, segs, e, ee, gw, bm, sstart, sbase, lane);
        else
          acc += pivot_pass<kPivotGlobal, true>(prow, pd, 0, 0, 0, segs, e, ee, gw, bm, sstart, sbase, lane);
      }
    }
    e = ee;
    if (e < e1) b = next_row(r_rp, H, b, e, lane);
  }
  return acc;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
  return v;
}

__device__ __forceinline__ unsigned long long dispatch_unit(const DevTask& tk, uint32_t unit, uint32_t* bm,
                                                            uint32_t* sstart, uint32_t* sbase, uint32_t lane,
                                                            uint32_t bm_words, uint32_t* err, uint32_t dbg) {
  if (tk.kind == kFusedRow) return fused_unit(tk, unit, bm, sstart, sbase, lane, bm_words);
  return task_unit(tk, unit, bm, sstart, sbase, lane, bm_words, err, dbg);
}

// Persistent form: every warp claims units from one head until the queue is
// empty.  MINB is the register budget's occupancy target (blocks per SM).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_count_queue(const DevTask* __restrict__ tasks,
                                                        const uint32_t* __restrict__ prefix, uint32_t ntasks,
                                                        uint32_t total_units, uint32_t* __restrict__ head,
                                                        unsigned long long* __restrict__ outs, uint32_t bm_words,
                                                        uint32_t dbg) {
  extern __shared__ __align__(16) uint32_t sh[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* bm = sh + warp * (bm_words + kSegWords);
  uint32_t* sstart = bm + bm_words;
  uint32_t* sbase = sstart + 33;
  uint32_t* err = head + 1;  // set when a staging copy gave up
  for (uint32_t i = lane; i < bm_words; i += 32) bm[i] = 0;
  staging_init(bm, bm_words, lane);
  while (true) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(head, 1u);
    g = __shfl_sync(FULL, g, 0);
    if (g >= total_units) break;
    uint32_t lo = 0, hi = ntasks;  // last t with prefix[t] <= g
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (prefix[mid] <= g) lo = mid; else hi = mid;
    }
    const DevTask& tk = tasks[lo];
    const unsigned long long c =
        warp_sum(dispatch_unit(tk, g - prefix[lo], bm, sstart, sbase, lane, bm_words, err, dbg));
    if (lane == 0 && c) atomicAdd(&outs[tk.slot], c);
    if (staging_dead(bm, bm_words)) break;
  }
}

// Plain form: one task per launch; warps stride over the task's units.
__global__ void __launch_bounds__(256, 4) k_count_task(const DevTask* __restrict__ task, uint32_t units,
                                                       unsigned long long* __restrict__ outs, uint32_t bm_words,
                                                       uint32_t* __restrict__ err, uint32_t dbg) {
  extern __shared__ __align__(16) uint32_t sh[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* bm = sh + warp * (bm_words + kSegWords);
  uint32_t* sstart = bm + bm_words;
  uint32_t* sbase = sstart + 33;
  for (uint32_t i = lane; i < bm_words; i += 32) bm[i] = 0;
  staging_init(bm, bm_words, lane);
  const DevTask& tk = *task;
  const uint32_t wpb = blockDim.x >> 5;
  unsigned long long acc = 0;
  for (uint32_t u = blockIdx.x * wpb + warp; u < units; u += gridDim.x * wpb) {
    acc += dispatch_unit(tk, u, bm, sstart, sbase, lane, bm_words, err, dbg);
    if (staging_dead(bm, bm_words)) break;
  }
  acc = warp_sum(acc);
  if (lane == 0 && acc) atomicAdd(&outs[tk.slot], acc);
}

// Fused persistent form.  A unit's loop state lives in a per-warp frame in
// shared memory while the probe loop runs, so the loop keeps the whole
// register budget (the persistent kernel runs at 40 registers per thread to
// keep 48 warps per SM resident; state held in registers across the probe
// loop would spill to local memory, which misses the small L1 left beside
// the bitmaps).  Lane 0 writes the frame; every lane reads it back after a
// __syncwarp.
struct FusedFrame {
  const uint32_t* rp;    // reversed tile (j, i): row pointers
  const uint2* rec;      // its forward-edge records
  const uint4* desc;     // per vertex: row start, pair start, first id, last id
  const uint32_t* gi;    // oriented CSR ids
  const uint2* gw;       // word-compressed rows
  uint32_t H, e1, b, ee; // rows, unit end, current row, end of the current row's entries
  uint32_t pivot_base, ps, pd, base, words, rlen, kind, slot;
  uint32_t ws, wn;       // the pivot row's word pairs
  uint32_t mask0;        // bits kept of the first pair (pivot_suffix)
};
static_assert(sizeof(FusedFrame) <= (kSegWords - kFrameOffset) * sizeof(uint32_t), "frame does not fit");

enum : uint32_t { kNoPivot = 0xffffffffu };

// Choose the pivot structure of row v (ids prow[0..pd)) and record it in the frame.
// first / last: the row's first and last id.
__device__ __forceinline__ void fused_choose(volatile FusedFrame* fr, const uint32_t* __restrict__ prow, uint32_t pd,
                                             uint32_t wn, uint32_t first, uint32_t last, uint32_t bm_words,
                                             uint32_t lane) {
  uint32_t kind = kNoPivot, base = 0, words = 0, rlen = 0;
  if (pd > 0) {
    const uint32_t span_words = (last >> 5) - (first >> 5) + 1;
    if (span_words < bm_words) {
      kind = kPivotBitmap;
      base = first & ~31u;  // word-aligned: a streamed pair meets exactly one bitmap word
      words = span_words;
    } else {
      // a wide row: a rank bitmap when its block entries (2 words per 32
      // words of span) and masks (1 per pair) fit the buffer
      const uint32_t blocks = (span_words + 31) >> 5;
      if (2 * blocks + wn <= bm_words) {
        kind = kPivotRank;
        base = first >> 5;  // first word
        words = blocks;
        rlen = span_words;
      }
    }
    if (kind == kNoPivot && span_words >= bm_words) {
      // bitmap over the top words of the row, the few ids below them in a short list
      const uint32_t wwords = bm_words - 1 - kSplitList;
      const uint32_t wbase = ((last >> 5) - (wwords - 1)) << 5;
      rlen = lower_bound_u32(prow, pd, wbase);
      if (rlen <= kSplitList) {
        kind = kPivotSplit;
        base = wbase;
        words = wwords;
      } else {
        kind = pd <= bm_words ? kPivotList : kPivotGlobal;
        rlen = 0;
      }
    }
  }
  if (lane == 0) {
    fr->pd = pd;
    fr->kind = kind;
    fr->base = base;
    fr->words = words;
    fr->rlen = rlen;
  }
}

template <uint32_t KIND>
__device__ __forceinline__ void fused_build(const uint32_t* __restrict__ prow, uint32_t pd, uint32_t base,
                                            uint32_t rlen, uint32_t* bm, uint32_t* res, uint32_t lane) {
  if constexpr (KIND == kPivotBitmap) {
    for (uint32_t i = lane; i < pd; i += 32) {
      const uint32_t y = prow[i] - base;
      atomicOr(&bm[y >> 5], 1u << (y & 31));
    }
  } else if constexpr (KIND == kPivotSplit) {
    for (uint32_t i = lane; i < pd; i += 32) {
      const uint32_t x = prow[i];
      if (i < rlen) {
        res[i] = x;
      } else {
        const uint32_t y = x - base;
        atomicOr(&bm[y >> 5], 1u << (y & 31));
      }
    }
  } else if constexpr (KIND == kPivotList) {
    for (uint32_t i = lane; i < pd; i += 32) bm[i] = prow[i];
  }
}

// Bitmap of a pivot row from its word pairs: one plain store per 32-id word
// (a row holds each word once), where setting the bits id by id took one
// shared-memory atomic per id, serialised on the words that several ids
// share.  Split kind: only the words of its window (w >= base_w).
template <uint32_t KIND>
__device__ __forceinline__ void fused_build_words(const uint2* __restrict__ pw, uint32_t wn, uint32_t base_w,
                                                  uint32_t mask0, uint32_t* bm, uint32_t lane) {
  for (uint32_t i = lane; i < wn; i += 32) {
    const uint2 w = pw[i];
    if (KIND == kPivotBitmap || w.x >= base_w) bm[w.x - base_w] = i == 0 ? (w.y & mask0) : w.y;
  }
}

// Rank pivot from its word pairs (first word fw, `blocks` entries of 32
// words): pair i sets its presence bit, and the first pair of each block
// writes its own index as the block's base; masks land in pair order (a
// row's words strictly increase, so a word's rank is its pair index).
__device__ __forceinline__ void fused_build_rank(const uint2* __restrict__ pw, uint32_t wn, uint32_t mask0,
                                                 uint32_t fw, uint32_t blocks, uint32_t* bm, uint32_t lane) {
  uint32_t* masks = bm + 2 * blocks;
  for (uint32_t c = 0; c < wn; c += 32) {  // every lane runs every round: the shuffle needs them all
    const uint32_t i = c + lane;
    const uint2 w = i < wn ? pw[i] : make_uint2(fw, 0u);
    uint32_t prev = __shfl_up_sync(FULL, w.x, 1);  // the previous pair's word, from the lane before
    if (lane == 0 && c > 0) prev = pw[c - 1].x;
    if (i < wn) {
      const uint32_t rel = w.x - fw;
      const uint32_t blk = rel >> 5;
      atomicOr(&bm[2 * blk], 1u << (rel & 31));
      if (i == 0 || ((prev - fw) >> 5) != blk) bm[2 * blk + 1] = i;
      masks[i] = i == 0 ? (w.y & mask0) : w.y;
    }
  }
}

// Back to zero: the entries of the blocks that hold a pair, and the masks.
__device__ __forceinline__ void fused_clear_rank(const uint2* __restrict__ pw, uint32_t wn, uint32_t fw,
                                                 uint32_t blocks, uint32_t* bm, uint32_t lane) {
  uint32_t* masks = bm + 2 * blocks;
  for (uint32_t i = lane; i < wn; i += 32) {
    const uint32_t blk = (pw[i].x - fw) >> 5;
    bm[2 * blk] = 0;
    bm[2 * blk + 1] = 0;
    masks[i] = 0;
  }
}

template <uint32_t KIND>
__device__ __forceinline__ void fused_clear_words(const uint2* __restrict__ pw, uint32_t wn, uint32_t base_w,
                                                  uint32_t words, uint32_t* bm, uint32_t lane) {
  // a bitmap with at least a third of its words set (or a split window as
  // many words as the row has pairs) is cleared as a range, stores only;
  // otherwise the row's words are read again and cleared one by one
  if ((KIND == kPivotBitmap && 3 * wn >= words) || wn >= words) {
    for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
  } else {
    for (uint32_t i = lane; i < wn; i += 32) {
      const uint32_t x = pw[i].x;
      if (KIND == kPivotBitmap || x >= base_w) bm[x - base_w] = 0;
    }
  }
}

template <uint32_t KIND>
__device__ __forceinline__ void fused_clear(const uint32_t* __restrict__ prow, uint32_t pd, uint32_t base,
                                            uint32_t words, uint32_t rlen, uint32_t* bm, uint32_t* res,
                                            uint32_t lane) {
  // up to 512 words are cleared as a range (16 stores a lane, no loads);
  // beyond that, the words of the row's ids, read again
  if constexpr (KIND == kPivotBitmap) {
    if (words <= 512 || pd >= words) {
      for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
    } else {
      for (uint32_t i = lane; i < pd; i += 32) bm[(prow[i] - base) >> 5] = 0;
    }
  } else if constexpr (KIND == kPivotSplit) {
    if (pd - rlen >= words) {
      for (uint32_t i = lane; i < words; i += 32) bm[i] = 0;
    } else {
      for (uint32_t i = lane + rlen; i < pd; i += 32) bm[(prow[i] - base) >> 5] = 0;
    }
    for (uint32_t i = lane; i < rlen; i += 32) res[i] = 0;
  } else if constexpr (KIND == kPivotList) {
    for (uint32_t i = lane; i < pd; i += 32) bm[i] = 0;
  }
}

// Probe entries [e, ee) of the frame's rows tile against the built pivot of kind KIND.
template <uint32_t KIND>
__device__ __forceinline__ uint32_t fused_probe(volatile FusedFrame* fr, const uint32_t* __restrict__ prow,
                                                uint32_t e, uint32_t ee, uint32_t* bm, uint32_t* sstart,
                                                uint32_t* sbase, uint32_t bm_words, uint32_t lane) {
  PivotView pv;
  pv.row = prow;
  pv.len = fr->pd;
  pv.base = fr->base;
  pv.cap = KIND == kPivotRank ? fr->rlen : fr->words * 32;
  pv.first = KIND == kPivotBitmap || KIND == kPivotRank ? 0u : prow[0];
  pv.last = KIND == kPivotBitmap || KIND == kPivotRank ? 0u : prow[pv.len - 1];
  pv.res = KIND == kPivotRank ? bm + 2 * fr->words : bm + fr->words + 1;
  pv.rlen = fr->rlen;
  const RecSegs segs{(const uint2*)fr->rec};
  return probe_entries<KIND, true>(segs, e, ee, reinterpret_cast<const uint32_t*>(fr->gw), bm, sstart, sbase, pv,
                                   lane);
}

// Pivots too wide for a span bitmap (split, list, global kinds): a separate
// function, so their register needs do not weigh on the common bitmap path.
__device__ __noinline__ uint32_t fused_wide(volatile FusedFrame* fr, uint32_t kind, const uint32_t* prow, uint32_t e,
                                            uint32_t ee, uint32_t* bm, uint32_t* sstart, uint32_t* sbase,
                                            uint32_t bm_words, uint32_t lane) {
  uint32_t* res = bm + fr->words + 1;
  if (kind == kPivotSplit) {
    const uint32_t rlen = fr->rlen;
    for (uint32_t i = lane; i < rlen; i += 32) res[i] = prow[i];
    fused_build_words<kPivotSplit>((const uint2*)fr->gw + fr->ws, fr->wn, fr->base >> 5, fr->mask0, bm, lane);
    __syncwarp();
    return fused_probe<kPivotSplit>(fr, prow, e, ee, bm, sstart, sbase, bm_words, lane);
  }
  if (kind == kPivotList) {
    fused_build<kPivotList>(prow, fr->pd, 0, 0, bm, res, lane);
    __syncwarp();
    return fused_probe<kPivotList>(fr, prow, e, ee, bm, sstart, sbase, bm_words, lane);
  }
  __syncwarp();
  return fused_probe<kPivotGlobal>(fr, prow, e, ee, bm, sstart, sbase, bm_words, lane);
}

template <int MINB>
__global__ void __launch_bounds__(256, MINB) k_fused_queue(const DevTask* __restrict__ tasks,
                                                        const uint32_t* __restrict__ prefix, uint32_t ntasks,
                                                        uint32_t total_units, uint32_t* __restrict__ head,
                                                        unsigned long long* __restrict__ outs, uint32_t bm_words) {
  extern __shared__ __align__(16) uint32_t sh[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* bm = sh + warp * (bm_words + kSegWords);
  uint32_t* sstart = bm + bm_words;
  uint32_t* sbase = sstart + 33;
  volatile FusedFrame* fr = reinterpret_cast<volatile FusedFrame*>(bm + bm_words + kFrameOffset);
  for (uint32_t i = lane; i < bm_words; i += 32) bm[i] = 0;
  __syncwarp();
  while (true) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(head, 1u);
    g = __shfl_sync(FULL, g, 0);
    if (g >= total_units) break;
    uint32_t lo = 0, hi = ntasks;  // last t with prefix[t] <= g
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (prefix[mid] <= g) lo = mid; else hi = mid;
    }
    const uint32_t first_unit = prefix[lo];
    if (lane == 0) {
      const DevTask* tk = tasks + lo;
      const uint32_t e0 = (g - first_unit) * tk->unit_edges;  // < nnz < 2^32
      const uint32_t nnz = tk->rows.nnz;
      fr->rp = tk->rows.rp;
      fr->rec = tk->rows.rec;
      fr->desc = tk->g_desc;
      fr->gi = tk->g_indices;
      fr->gw = tk->g_words;
      fr->H = tk->rows.H;
      fr->e1 = nnz - e0 > tk->unit_edges ? e0 + tk->unit_edges : nnz;
      fr->b = tk->rows.erow[e0 >> 5];  // units start at multiples of 32 entries
      fr->ee = e0;
      fr->pivot_base = tk->pivot_base;
      fr->slot = tk->slot;
    }
    __syncwarp();
    unsigned long long acc = 0;
    while (true) {
      const uint32_t e = fr->ee;
      if (e >= fr->e1) break;
      // row b's entries in this unit and its pivot row N+(v), v = pivot_base + b
      {
        const uint32_t b = fr->b;
        const uint32_t ee = min(fr->rp[b + 1], fr->e1);
        const uint32_t lo = fr->pivot_base;
        const uint32_t v = lo + b;
        const uint32_t* gi = fr->gi;
        // the pivot row's extent in one pair of 16-byte loads
        const uint4 d0 = fr->desc[v], d1 = fr->desc[v + 1];
        uint32_t ps = d0.x, pd = d1.x - d0.x, ws = d0.y, wn = d1.y - d0.y;
        uint32_t first = d0.z;
        uint32_t mask0 = FULL;
        // ids of N+(v) below the task columns (never, for a CSR oriented from
        // lower to higher ids) are left out of the pivot
        if (pd > 0 && first < lo) {
          pivot_suffix(gi, (const uint2*)fr->gw, lo, ps, pd, ws, wn, mask0);
          if (pd > 0) first = gi[ps];
        }
        fused_choose(fr, gi + ps, pd, wn, first, d0.w, bm_words, lane);
        if (lane == 0) {
          fr->ee = ee;
          fr->ps = ps;
          fr->ws = ws;
          fr->wn = wn;
          fr->mask0 = mask0;
        }
        __syncwarp();
      }
      const uint32_t kind = fr->kind;
      if (kind != kNoPivot) {
        const uint32_t* prow = fr->gi + fr->ps;
        const uint32_t ee = fr->ee;
        uint32_t* res = bm + fr->words + 1;
        switch (kind) {
          case kPivotBitmap:
            fused_build_words<kPivotBitmap>((const uint2*)fr->gw + fr->ws, fr->wn, fr->base >> 5, fr->mask0, bm,
                                            lane);
            __syncwarp();
            acc += fused_probe<kPivotBitmap>(fr, prow, e, ee, bm, sstart, sbase, bm_words, lane);
            break;
          case kPivotRank:
            fused_build_rank((const uint2*)fr->gw + fr->ws, fr->wn, fr->mask0, fr->base, fr->words, bm, lane);
            __syncwarp();
            acc += fused_probe<kPivotRank>(fr, prow, e, ee, bm, sstart, sbase, bm_words, lane);
            break;
          default:
            acc += fused_wide(fr, kind, prow, e, ee, bm, sstart, sbase, bm_words, lane);
        }
        __syncwarp();
        // the buffer returns to all-zero for the next pivot, whatever its kind
        {
          const uint32_t* prow2 = fr->gi + fr->ps;
          uint32_t* res2 = bm + fr->words + 1;
          const uint2* pw = (const uint2*)fr->gw + fr->ws;
          switch (fr->kind) {
            case kPivotBitmap: fused_clear_words<kPivotBitmap>(pw, fr->wn, fr->base >> 5, fr->words, bm, lane); break;
            case kPivotRank: fused_clear_rank(pw, fr->wn, fr->base, fr->words, bm, lane); break;
            case kPivotSplit: {
              fused_clear_words<kPivotSplit>(pw, fr->wn, fr->base >> 5, fr->words, bm, lane);
              const uint32_t rlen = fr->rlen;
              for (uint32_t i = lane; i < rlen; i += 32) res2[i] = 0;
              break;
            }
            case kPivotList: fused_clear<kPivotList>(prow2, fr->pd, 0, 0, 0, bm, res2, lane); break;
            default: break;
          }
        }
        __syncwarp();
      }
      const uint32_t e2 = fr->ee;
      if (e2 < fr->e1) {
        const uint32_t nb = next_row(fr->rp, fr->H, fr->b, e2, lane);
        if (lane == 0) fr->b = nb;
      }
      __syncwarp();
    }
    const unsigned long long c = warp_sum(acc);
    if (lane == 0 && c) atomicAdd(&outs[fr->slot], c);
  }
}

size_t smem_bytes(uint32_t bm_words, uint32_t warps) {
  return (size_t)warps * (bm_words + kSegWords) * sizeof(uint32_t);
}

uint32_t norm_bm_words(uint32_t w) {
  if (w == 0) w = 1024;
  w = (w + 3) & ~3u;
  return std::max<uint32_t>(w, 2 * kSplitList);
}

uint32_t norm_warps(uint32_t w) { return w == 0 ? 8 : std::min<uint32_t>(std::max<uint32_t>(w, 1), 8); }

}  // namespace

size_t smem_bytes_for(const bbtc_opts& o) {
  return smem_bytes(norm_bm_words(o.bitmap_words), norm_warps(o.warps_per_block));
}

int kernel_smem_optin(bbtc_ctx* ctx, const bbtc_opts& o) {
  const size_t sm = smem_bytes(norm_bm_words(o.bitmap_words), norm_warps(o.warps_per_block));
  if (sm > ctx->smem_optin)
    return fail(BBTC_ERR_ARG, "bitmap_words x warps_per_block needs " + std::to_string(sm) +
                                  " bytes of shared memory; the device allows " + std::to_string(ctx->smem_optin));
  if (sm <= ctx->smem_set) return BBTC_OK;
  BBTC_CUDA(cudaFuncSetAttribute(k_count_queue<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_count_queue<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_count_queue<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_fused_queue<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_fused_queue<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_fused_queue<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_fused_queue<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_count_task, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  ctx->smem_set = sm;
  return BBTC_OK;
}

// Average out-row length of row part i over its tiles (for unit sizing).
static double part_row_len(const bbtc_graph* g, uint32_t i) {
  uint64_t z = 0;
  uint32_t rows = 1;
  for (uint32_t k = 0; k < g->P; k++) {
    z += g->rev.nnz[k * g->P + i];  // reversed tile (k, i) holds the edges of forward tile (i, k)
    if (g->fwd_built) rows = std::max(rows, g->fwd.nerows[i * g->P + k]);
  }
  if (!g->fwd_built) rows = std::max<uint32_t>(1, g->cuts[i + 1] - g->cuts[i]);
  return (double)z / rows;
}

// Build the device task array for a request.  A single graph keeps the
// caller's task order (its border split); several graphs are merged into one
// queue ordered by estimated probe work, heaviest first.  With `fused`, every
// graph's full task list runs as task rows (i, j).
static int make_plan(const std::vector<bbtc_graph*>& graphs, const std::vector<std::vector<bbtc_task>>& tasks,
                     const bbtc_opts& o, bool fused, Plan* plan) {
  const uint32_t bmw = norm_bm_words(o.bitmap_words);
  // default unit size: task rows of the fused form run as 32-entry units
  // (below); explicit task lists as units of ~8192 probes
  const uint32_t unit_work = o.unit_work ? o.unit_work : (fused ? 256 : 8192);
  std::vector<DevTask> list;
  std::vector<double> cost;
  auto add = [&](DevTask d, double avg_probe) {
    uint32_t K = (uint32_t)std::min(16384.0, std::max(32.0, unit_work / std::max(1.0, avg_probe)));
    K = (K + 31) & ~31u;
    d.unit_edges = K;
    list.push_back(d);
    cost.push_back((double)d.rows.nnz * std::max(1.0, avg_probe));
  };
  for (size_t gi = 0; gi < graphs.size(); gi++) {
    const bbtc_graph* g = graphs[gi];
    const uint32_t P = g->P;
    if (fused) {
      for (uint32_t i = 0; i < P; i++)
        for (uint32_t j = i; j < P; j++) {
          if (!g->rev.nnz[j * P + i]) continue;  // forward tile (i, j) is empty
          DevTask d{};
          d.rows = dev_tile(g->rev, g->cuts, j, i);
          d.kind = kFusedRow;
          d.slot = (uint32_t)gi;
          d.g_indptr = g->d_indptr;
          d.g_indices = g->d_indices;
          d.g_words = reinterpret_cast<const uint2*>(g->d_words);
          d.g_wptr = g->d_wptr;
          d.g_desc = static_cast<const uint4*>(g->d_desc);
          d.pivot_base = g->cuts[j];
          add(d, 0.5 * part_row_len(g, i));
          if (!o.unit_work) list.back().unit_edges = 0;  // set below from the request's size
        }
      continue;
    }
    for (const bbtc_task& t : tasks[gi]) {
      if (t.ab >= P * P || t.bc >= P * P || t.ac >= P * P)
        return fail(BBTC_ERR_ARG, "task names a tile outside the P x P grid");
      const uint32_t i = t.ab / P, j = t.ab % P, k = t.bc % P;
      if (t.bc / P != j || t.ac != i * P + k)
        return fail(BBTC_ERR_ARG, "task tiles are not of the form (i,j), (j,k), (i,k)");
      if (!g->fwd.nnz[t.ab] || !g->fwd.nnz[t.bc] || !g->fwd.nnz[t.ac]) continue;  // bb_tc.cpp:86-91
      DevTask d{};
      const bool u_centric = (o.kernel == BBTC_KERNEL_MERGE);
      if (u_centric) {
        d.rows = dev_tile(g->fwd, g->cuts, i, j);
        d.pivot = dev_tile(g->fwd, g->cuts, i, k);
        d.probe = dev_tile(g->fwd, g->cuts, j, k);
      } else {
        d.rows = dev_tile(g->rev, g->cuts, j, i);
        d.pivot = dev_tile(g->fwd, g->cuts, j, k);
        d.probe = dev_tile(g->fwd, g->cuts, i, k);
      }
      d.words = (d.pivot.W + 31) / 32;
      const bool fits_bitmap = d.words < bmw;  // the word after the part stays zero
      const bool fits_list = d.pivot.maxdeg <= bmw;
      if (!u_centric && o.kernel != BBTC_KERNEL_SEARCH && fits_bitmap)
        d.kind = kPivotBitmap;
      else
        d.kind = fits_list ? kPivotList : kPivotGlobal;
      d.slot = (uint32_t)gi;
      const uint32_t probe_tile = u_centric ? j * P + k : i * P + k;
      const uint32_t probe_rows = std::max<uint32_t>(1, g->fwd.nerows[probe_tile]);
      add(d, (double)d.probe.nnz / probe_rows);
    }
  }
  if (fused && !o.unit_work) {
    // default units of the fused task rows: 32 in-edges (one probe batch), or
    // 64 when the request has 2^25 in-edges or more -- at R-MAT s22 (64 M)
    // 64 was 5 % faster, at s20 (16 M) 13 % slower (too few units per warp
    // to balance the tail)
    uint64_t entries = 0;
    for (const DevTask& d : list) entries += d.rows.nnz;
    const uint32_t K = entries >= (1ull << 25) ? 64 : 32;
    for (DevTask& d : list) d.unit_edges = K;
  }
  std::vector<uint32_t> order(list.size());
  for (uint32_t q = 0; q < order.size(); q++) order[q] = q;
  if (graphs.size() > 1 || fused)
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  plan->tasks.clear();
  plan->prefix.assign(1, 0);
  uint64_t total = 0;
  for (uint32_t q : order) {
    const DevTask& d = list[q];
    total += ((uint64_t)d.rows.nnz + d.unit_edges - 1) / d.unit_edges;  // 64-bit: nnz may be near 2^32
    if (total >= 0xffffffffull) return fail(BBTC_ERR_UNSUPPORTED, "more than 2^32 work units in one request");
    plan->tasks.push_back(d);
    plan->prefix.push_back((uint32_t)total);
  }
  plan->total_units = (uint32_t)total;
  plan->fused = fused;
  return BBTC_OK;
}

void Plan::release() {
  if (exec) cudaGraphExecDestroy(exec);
  if (d_tasks) cudaFreeAsync(d_tasks, stream);
  if (d_prefix) cudaFreeAsync(d_prefix, stream);
  exec = nullptr;
  d_tasks = nullptr;
  d_prefix = nullptr;
  cap = 0;
}

static int enqueue_launches(bbtc_ctx* ctx, Plan* plan, const bbtc_opts& o, uint64_t* d_outs, uint32_t nouts) {
  cudaStream_t s = ctx->stream;
  const uint32_t bmw = norm_bm_words(o.bitmap_words);
  const uint32_t wpb = norm_warps(o.warps_per_block);
  const size_t sm = smem_bytes(bmw, wpb);
  auto* outs = reinterpret_cast<unsigned long long*>(d_outs);
  BBTC_CUDA(cudaMemsetAsync(d_outs, 0, nouts * sizeof(uint64_t), s));
  BBTC_CUDA(cudaMemsetAsync(ctx->d_unit_counter, 0, 2 * sizeof(uint32_t), s));  // queue head, staging flag
  plan->launches = 0;
  const uint32_t ntasks = (uint32_t)plan->tasks.size();
  if (ntasks == 0) return BBTC_OK;
  if (o.mode == BBTC_MODE_PLAIN) {
    for (uint32_t t = 0; t < ntasks; t++) {
      const uint32_t units = plan->prefix[t + 1] - plan->prefix[t];
      const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>((units + wpb - 1) / wpb, ctx->sms * 8));
      k_count_task<<<grid, wpb * 32, sm, s>>>(plan->d_tasks + t, units, outs, bmw, ctx->d_unit_counter + 1,
                                              ctx->debug_stage_polls);
      BBTC_CUDA(cudaGetLastError());
      plan->launches++;
    }
  } else {
    // the register budget: 4, 5, 6 or 8 resident blocks per SM (the per-task
    // queue kernel has no 5-block variant and runs 4 there)
    const uint32_t occ = o.occupancy >= 8 ? 8 : (o.occupancy >= 6 ? 6 : (o.occupancy == 5 ? 5 : 4));
    auto* fkern = occ == 8 ? k_fused_queue<8>
                           : (occ == 6 ? k_fused_queue<6> : (occ == 5 ? k_fused_queue<5> : k_fused_queue<4>));
    auto* qkern = occ == 8 ? k_count_queue<8> : (occ == 6 ? k_count_queue<6> : k_count_queue<4>);
    int per_sm = 0;
    if (plan->fused)
      BBTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fkern, wpb * 32, sm));
    else
      BBTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, qkern, wpb * 32, sm));
    per_sm = std::max(1, per_sm);
    if (o.blocks_per_sm) per_sm = std::min<int>(per_sm, (int)o.blocks_per_sm);
    // no more blocks than the queue has units for a warp each (a small batch
    // leaves the rest of the GPU to other streams)
    const uint64_t want = ((uint64_t)plan->total_units + wpb - 1) / wpb;
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)ctx->sms * per_sm, want));
    if (plan->fused)
      fkern<<<grid, wpb * 32, sm, s>>>(plan->d_tasks, plan->d_prefix, ntasks, plan->total_units,
                                       ctx->d_unit_counter, outs, bmw);
    else
      qkern<<<grid, wpb * 32, sm, s>>>(plan->d_tasks, plan->d_prefix, ntasks, plan->total_units,
                                       ctx->d_unit_counter, outs, bmw, ctx->debug_stage_polls);
    BBTC_CUDA(cudaGetLastError());
    plan->launches = 1;
  }
  return BBTC_OK;
}

int staging_status(bbtc_ctx* ctx) {
  uint32_t* h = reinterpret_cast<uint32_t*>(ctx->h_stage + kStageBad);
  BBTC_CUDA(cudaMemcpyAsync(h, ctx->d_unit_counter + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  BBTC_CUDA(cudaStreamSynchronize(ctx->stream));
  if (*h) return fail(BBTC_ERR_TIMEOUT, "a shared-memory staging copy did not complete; the count is void");
  return BBTC_OK;
}

// Options left at 0 ("auto") resolved for the request's graphs.  The
// bitmap: 1024 words per warp.  Rows wider than that run as rank bitmaps,
// so a larger buffer only costs occupancy (one B200, ms per count, 512 / 768
// / 1024 / 1536 / 2048 words: R-MAT s22 7.92 / 7.63 / 7.49 / 8.16 / 9.56;
// s24 - / - / 41.8 / 46.5 / 56.5).  Occupancy: fused task rows 6 blocks per
// SM (40 registers) while the bitmap leaves shared memory for them, else 4
// (64 registers); per-task kernels 4 (R-MAT s20: bitmap 10.4 ms at 4 against
// 12.4 at 6, search 14.4 / 15.7, merge 27.5 / 31.5).
static bbtc_opts resolve_opts(const std::vector<bbtc_graph*>& graphs, const bbtc_opts& in, bool fused) {
  bbtc_opts o = in;
  (void)graphs;
  if (!o.bitmap_words) o.bitmap_words = 1024;
  if (!o.occupancy) o.occupancy = fused && norm_bm_words(o.bitmap_words) <= 1024 ? 6 : 4;
  return o;
}

int count_enqueue(bbtc_ctx* ctx, const std::vector<bbtc_graph*>& graphs,
                  const std::vector<std::vector<bbtc_task>>& tasks, const bbtc_opts& in, bool fused,
                  uint64_t* d_outs, Plan* plan, bool reuse) {
  Range range("bbtc count enqueue");
  cudaStream_t s = ctx->stream;
  const bbtc_opts o = resolve_opts(graphs, in, fused);
  BBTC_TRY(kernel_smem_optin(ctx, o));
  if (!reuse) {
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
    BBTC_TRY(make_plan(graphs, tasks, o, fused, plan));
    const size_t nt = plan->tasks.size();
    if (nt) {
      if (nt > plan->cap || plan->stream != s) {
        plan->release();
        plan->stream = s;
        const size_t cap = std::max<size_t>(nt, 256);
        if (dev_malloc(&plan->d_tasks, cap * sizeof(DevTask), s) != cudaSuccess ||
            dev_malloc(&plan->d_prefix, (cap + 1) * sizeof(uint32_t), s) != cudaSuccess) {
          cudaGetLastError();
          plan->release();
          return fail(BBTC_ERR_NOMEM, "device allocation of the task queue failed");
        }
        plan->cap = cap;
      }
      // upload from the context's pinned staging (a pageable copy would go
      // through the driver's shared staging buffers, which other threads'
      // copies hold); the context keeps it across plans, since pinning host
      // memory can take milliseconds
      const size_t tb = nt * sizeof(DevTask), pb = (nt + 1) * sizeof(uint32_t);
      if (ctx->h_plan_done) BBTC_CUDA(cudaEventSynchronize(ctx->h_plan_done));  // the last upload has read it
      if (tb + pb > ctx->h_plan_cap) {
        if (ctx->h_plan) cudaFreeHost(ctx->h_plan);
        ctx->h_plan = nullptr;
        ctx->h_plan_cap = 0;
        const size_t want = std::max<size_t>(tb + pb, 64 << 10) * 2;
        BBTC_CUDA(cudaMallocHost(&ctx->h_plan, want));
        ctx->h_plan_cap = want;
      }
      if (!ctx->h_plan_done) BBTC_CUDA(cudaEventCreateWithFlags(&ctx->h_plan_done, cudaEventDisableTiming));
      std::memcpy(ctx->h_plan, plan->tasks.data(), tb);
      std::memcpy(ctx->h_plan + tb, plan->prefix.data(), pb);
      BBTC_CUDA(cudaMemcpyAsync(plan->d_tasks, ctx->h_plan, tb, cudaMemcpyHostToDevice, s));
      BBTC_CUDA(cudaMemcpyAsync(plan->d_prefix, ctx->h_plan + tb, pb, cudaMemcpyHostToDevice, s));
      BBTC_CUDA(cudaEventRecord(ctx->h_plan_done, s));
    }
    plan->captured = false;
  }
  if (plan->stage_polls != ctx->debug_stage_polls && plan->exec) {  // the launches take it as an argument
    cudaGraphExecDestroy(plan->exec);
    plan->exec = nullptr;
    plan->captured = false;
  }
  plan->stage_polls = ctx->debug_stage_polls;
  // A plan's first count launches directly: capturing and instantiating a
  // graph costs more host time than one launch, and pays only on replays,
  // so the capture waits for the plan's second count.
  if (!o.use_cuda_graph || !reuse) return enqueue_launches(ctx, plan, o, d_outs, (uint32_t)graphs.size());
  if (!plan->captured) {
    cudaGraph_t graph = nullptr;
    BBTC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_launches(ctx, plan, o, d_outs, (uint32_t)graphs.size());
    const cudaError_t ec = cudaStreamEndCapture(s, &graph);
    if (rc != BBTC_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return cuda_fail(ec, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&plan->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
    plan->captured = true;
  }
  BBTC_CUDA(cudaGraphLaunch(plan->exec, s));
  return BBTC_OK;
}

// ---- counting without allocation --------------------------------------------
//
// bbtc_count_csr_noalloc counts the triangles of an oriented CSR that the
// caller already holds in device memory, for callers that cannot allocate
// device memory themselves or through this library: code that runs inside
// another framework's device-memory manager (which owns the device's memory
// and hands out only slices of its own pool), processes held to a fixed
// device-memory quota, and paths that must not pay cudaMalloc / cudaFree's
// implicit device synchronisation.  It is the persistent queue kernel's
// scheme run over the CSR as one task (P = 1, the reference's row order: the
// pivot is N+(u), the rows streamed are N+(v) for v in N+(u)); every word of
// scratch -- the queue head, an error word, the total and one partial count
// per work unit -- lives in the static array below, so the call allocates
// nothing.  Limit: at most kNoAllocMaxEdges oriented edges.
constexpr uint32_t kNoAllocUnitEdges = 256;
constexpr uint64_t kNoAllocMaxEdges = 1ull << 24;  // 16,777,216 oriented edges
constexpr uint32_t kNoAllocMaxUnits = (uint32_t)(kNoAllocMaxEdges / kNoAllocUnitEdges);

struct NoAllocScratch {
  uint32_t head;   // next work unit
  uint32_t error;  // bit 0: a row pointer or id outside the CSR was met
  unsigned long long total;
  uint32_t pad[60];
  unsigned long long partial[kNoAllocMaxUnits];
};

// One copy per device that loads the library, kept until the process exits
// (about 512 KiB).  Host code must not take its address directly: the
// device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

namespace {

// Row ranges of a caller CSR, checked against [0, m] and ids against n.
struct CheckedCsrSegs {
  const uint32_t* __restrict__ col;
  const uint32_t* __restrict__ rp;
  uint32_t n;
  uint64_t m;
  uint32_t* err;
  __device__ __forceinline__ void get(uint32_t q, uint32_t& start, uint32_t& len) const {
    const uint32_t v = col[q];
    start = 0;
    len = 0;
    if (v >= n) {
      atomicOr(err, 1u);
      return;
    }
    const uint32_t a = rp[v], b = rp[v + 1];
    if (b < a || (uint64_t)b > m) {
      atomicOr(err, 1u);
      return;
    }
    start = a;
    len = b - a;
  }
};

__global__ void __launch_bounds__(256, 4) k_count_csr_static(const uint32_t* __restrict__ indptr,
                                                             const uint32_t* __restrict__ indices, uint32_t n,
                                                             uint64_t m, uint32_t units, NoAllocScratch* scr,
                                                             uint32_t bm_words) {
  extern __shared__ __align__(16) uint32_t sh[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* bm = sh + warp * (bm_words + kSegWords);
  uint32_t* sstart = bm + bm_words;
  uint32_t* sbase = sstart + 33;
  for (uint32_t i = lane; i < bm_words; i += 32) bm[i] = 0;
  __syncwarp();
  const CheckedCsrSegs segs{indices, indptr, n, m, &scr->error};
  while (true) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(&scr->head, 1u);
    g = __shfl_sync(FULL, g, 0);
    if (g >= units) break;
    const uint32_t e0 = g * kNoAllocUnitEdges;
    const uint64_t e1w = (uint64_t)e0 + kNoAllocUnitEdges;
    const uint32_t e1 = (uint32_t)(e1w < m ? e1w : m);
    uint32_t e = e0;
    uint32_t u = row_of(indptr, n, e);  // < n (the host refuses n == 0 with m > 0)
    unsigned long long acc = 0;
    while (e < e1) {
      if (u >= n) {  // no row ends after e: indptr[n] < m
        if (lane == 0) atomicOr(&scr->error, 1u);
        break;
      }
      const uint32_t a = indptr[u], b = indptr[u + 1];
      if (b < a || (uint64_t)b > m || b <= e) {  // malformed row pointers: stop this unit
        if (lane == 0) atomicOr(&scr->error, 1u);
        break;
      }
      const uint32_t ee = min(b, e1);
      const uint32_t pd = b - a;
      const uint32_t* prow = indices + a;
      // the caller's row must be strictly increasing: the bitmap is indexed by id
      bool sorted = true;
      for (uint32_t i = lane; i + 1 < pd; i += 32) sorted &= prow[i] < prow[i + 1];
      if (!__all_sync(FULL, sorted)) {
        if (lane == 0) atomicOr(&scr->error, 1u);
        e = ee;
        if (e < e1) u = next_row(indptr, n, u, e, lane);
        continue;
      }
      const uint32_t first = prow[0], last = prow[pd - 1];
      const uint32_t span_words = last >= first ? ((last - first) >> 5) + 1 : 0xffffffffu;
      if (span_words < bm_words)
        acc += pivot_pass<kPivotBitmap, false>(prow, pd, first, span_words, 0, segs, e, ee, indices, bm, sstart, sbase,
                                        lane);
      else if (pd <= bm_words)
        acc += pivot_pass<kPivotList, false>(prow, pd, 0, 0, 0, segs, e, ee, indices, bm, sstart, sbase, lane);
      else
        acc += pivot_pass<kPivotGlobal, false>(prow, pd, 0, 0, 0, segs, e, ee, indices, bm, sstart, sbase, lane);
      e = ee;
      if (e < e1) u = next_row(indptr, n, u, e, lane);
    }
    acc = warp_sum(acc);
    if (lane == 0) scr->partial[g] = acc;
  }
}

// total = sum of the unit partials, in a fixed order (one block).
__global__ void k_noalloc_total(NoAllocScratch* scr, uint32_t units) {
  __shared__ unsigned long long part[1024];
  unsigned long long s = 0;
  for (uint32_t i = threadIdx.x; i < units; i += blockDim.x) s += scr->partial[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (uint32_t w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) scr->total = part[0];
}

}  // namespace

namespace {

// Per device, set up by the first call on it: the device address of
// g_noalloc_scratch, the kernel's shared-memory attribute and its grid.
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};
uint32_t g_noalloc_grid[kMaxDevices] = {};

constexpr uint32_t kNoAllocBitmapWords = 1024, kNoAllocWarps = 8;

int noalloc_setup(int dev, void** ptr, uint32_t* grid) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    // the device is current: resolve the array's device address
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    const size_t sm = smem_bytes(kNoAllocBitmapWords, kNoAllocWarps);
    BBTC_CUDA(cudaFuncSetAttribute(k_count_csr_static, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    int sms = 0, per_sm = 0;
    BBTC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    BBTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_count_csr_static, kNoAllocWarps * 32, sm));
    g_noalloc_grid[dev] = (uint32_t)std::max(1, sms * std::max(1, per_sm));
    g_noalloc_ptr[dev] = p;
  }
  *ptr = g_noalloc_ptr[dev];
  *grid = g_noalloc_grid[dev];
  return BBTC_OK;
}

}  // namespace

}  // namespace bbtc

extern "C" int bbtc_count_csr_noalloc(const uint32_t* d_indptr, const uint32_t* d_indices, uint32_t n, uint64_t m,
                                      uint64_t* out, void* stream) {
  using namespace bbtc;
  if (!d_indptr || (m && !d_indices) || !out) return fail(BBTC_ERR_ARG, "NULL argument");
  if (n == 0xffffffffu) return fail(BBTC_ERR_ARG, "n must be below 2^32 - 1");
  if (n == 0 && m > 0) return fail(BBTC_ERR_ARG, "a CSR with no rows cannot hold edges (n == 0, m > 0)");
  if (m > kNoAllocMaxEdges)
    return fail(BBTC_ERR_CAPACITY, "bbtc_count_csr_noalloc takes at most " + std::to_string(kNoAllocMaxEdges) +
                                       " oriented edges (its static scratch has one slot per 256 edges); got " +
                                       std::to_string(m));
  int dev = 0;
  BBTC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= (int)kMaxDevices) return fail(BBTC_ERR_NODEV, "device index beyond the supported range");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  void* ptr = nullptr;
  uint32_t grid = 0;
  BBTC_TRY(noalloc_setup(dev, &ptr, &grid));
  NoAllocScratch* scr = static_cast<NoAllocScratch*>(ptr);
  // head, error and total start at zero; the partials of this call's units are all rewritten
  BBTC_CUDA(cudaMemsetAsync(scr, 0, offsetof(NoAllocScratch, pad), s));
  const uint32_t units = (uint32_t)((m + kNoAllocUnitEdges - 1) / kNoAllocUnitEdges);
  if (units > 0) {
    const size_t sm = smem_bytes(kNoAllocBitmapWords, kNoAllocWarps);
    k_count_csr_static<<<grid, kNoAllocWarps * 32, sm, s>>>(d_indptr, d_indices, n, m, units, scr,
                                                              kNoAllocBitmapWords);
    BBTC_CUDA(cudaGetLastError());
    k_noalloc_total<<<1, 1024, 0, s>>>(scr, units);
    BBTC_CUDA(cudaGetLastError());
  }
  struct {
    uint32_t head, error;
    unsigned long long total;
  } hdr{0, 0, 0};
  BBTC_CUDA(cudaMemcpyAsync(&hdr, scr, sizeof(hdr), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaStreamSynchronize(s));
  if (hdr.error) return fail(BBTC_ERR_INPUT, "the CSR has a row pointer or column id outside its bounds, or an "
                                            "unsorted row");
  *out = hdr.total;
  return BBTC_OK;
}

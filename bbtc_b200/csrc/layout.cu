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
//   * forward tiles (x, y): rows of part x, tile-local columns of part y --
//     the reference's tiles, used as ab / bc / ac;
//   * reversed tiles (y, x): the same edges grouped by their column vertex --
//     the CSC of forward tile (x, y), which the pivot-row kernels walk.
//
// Each non-empty tile owns a row-pointer segment of H+1 tile-local offsets
// (first entry 0) and a column segment of nnz ids; both start on a 16-byte
// boundary (multiples of 4 words) inside two pools.  Empty tiles own nothing.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "internal.h"

namespace bbtc {

namespace {

__device__ __forceinline__ uint32_t part_of(const uint32_t* cuts, uint32_t P, uint32_t u) {
  // largest x in [0, P) with cuts[x] <= u (skips empty parts); needs u < cuts[P]
  uint32_t lo = 0, hi = P;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (cuts[mid] <= u) lo = mid; else hi = mid;
  }
  return lo;
}

// Input contract check: monotone row pointers, strictly increasing rows, ids < n.
__global__ void k_validate(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                           uint32_t n, uint64_t m, uint32_t* __restrict__ bad) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
    if (u == 0 && indptr[0] != 0) atomicOr(bad, 1u);
    if (u == n - 1 && (uint64_t)indptr[n] != m) atomicOr(bad, 2u);
    const uint32_t a = indptr[u], b = indptr[u + 1];
    if (b < a || (uint64_t)b > m) {
      atomicOr(bad, 4u);
      continue;
    }
    int64_t prev = -1;
    for (uint32_t e = a; e < b; e++) {
      const uint32_t c = indices[e];
      if (c >= n) { atomicOr(bad, 8u); break; }
      if ((int64_t)c <= prev) { atomicOr(bad, 16u); break; }
      prev = c;
    }
  }
}

// Walk row u's entries as runs of one column part each; calls f(y, first, count).
template <class F>
__device__ __forceinline__ void for_each_run(const uint32_t* __restrict__ indices, uint32_t a, uint32_t b,
                                             const uint32_t* cuts, F&& f) {
  uint32_t y = 0;
  uint32_t e = a;
  while (e < b) {
    const uint32_t c = indices[e];
    while (c >= cuts[y + 1]) y++;
    const uint32_t hi = cuts[y + 1];
    uint32_t e2 = e + 1;
    while (e2 < b && indices[e2] < hi) e2++;
    f(y, e, e2 - e);
    e = e2;
  }
}

// Per-tile nnz, longest row and non-empty row count (CTA histograms in shared memory).
__global__ void k_tile_count(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                             uint32_t n, const uint32_t* __restrict__ cuts_g, uint32_t P,
                             uint32_t* __restrict__ nnz, uint32_t* __restrict__ maxdeg,
                             uint32_t* __restrict__ nerows) {
  extern __shared__ uint32_t sh[];
  const uint32_t T = P * P;
  uint32_t* h_nnz = sh;
  uint32_t* h_max = sh + T;
  uint32_t* h_ne = sh + 2 * T;
  uint32_t* cuts = sh + 3 * T;
  for (uint32_t t = threadIdx.x; t < 3 * T; t += blockDim.x) sh[t] = 0;
  for (uint32_t t = threadIdx.x; t <= P; t += blockDim.x) cuts[t] = cuts_g[t];
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
    const uint32_t x = part_of(cuts, P, u);
    const uint32_t a = indptr[u], b = indptr[u + 1];
    for_each_run(indices, a, b, cuts, [&](uint32_t y, uint32_t, uint32_t cnt) {
      const uint32_t t = x * P + y;
      atomicAdd(&h_nnz[t], cnt);
      atomicMax(&h_max[t], cnt);
      atomicAdd(&h_ne[t], 1u);
    });
  }
  __syncthreads();
  for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
    if (h_nnz[t]) {
      atomicAdd(&nnz[t], h_nnz[t]);
      atomicMax(&maxdeg[t], h_max[t]);
      atomicAdd(&nerows[t], h_ne[t]);
    }
  }
}

// rp_pool[rp_off[t] + r + 1] = length of row r in tile t.
__global__ void k_row_counts(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                             uint32_t n, const uint32_t* __restrict__ cuts_g, uint32_t P,
                             const uint64_t* __restrict__ rp_off, uint32_t* __restrict__ pool) {
  __shared__ uint32_t cuts[kMaxParts + 1];
  for (uint32_t t = threadIdx.x; t <= P; t += blockDim.x) cuts[t] = cuts_g[t];
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
    const uint32_t x = part_of(cuts, P, u);
    const uint32_t r = u - cuts[x];
    for_each_run(indices, indptr[u], indptr[u + 1], cuts, [&](uint32_t y, uint32_t, uint32_t cnt) {
      pool[rp_off[x * P + y] + r + 1] = cnt;
    });
  }
}

// After an inclusive scan over the whole pool, make each segment tile-local.
__global__ void k_localize(uint32_t* __restrict__ pool, uint64_t len, const uint64_t* __restrict__ seg_start,
                           const uint32_t* __restrict__ seg_base, uint32_t nseg) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < len; s += stride) {
    uint32_t lo = 0, hi = nseg;  // last q with seg_start[q] <= s
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (seg_start[mid] <= s) lo = mid; else hi = mid;
    }
    pool[s] -= seg_base[lo];
  }
}

__global__ void k_scatter(const uint32_t* __restrict__ indptr, const uint32_t* __restrict__ indices,
                          uint32_t n, const uint32_t* __restrict__ cuts_g, uint32_t P,
                          const uint64_t* __restrict__ rp_off, const uint64_t* __restrict__ col_off,
                          const uint32_t* __restrict__ rp_pool, uint32_t* __restrict__ col_pool) {
  __shared__ uint32_t cuts[kMaxParts + 1];
  for (uint32_t t = threadIdx.x; t <= P; t += blockDim.x) cuts[t] = cuts_g[t];
  __syncthreads();
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride) {
    const uint32_t x = part_of(cuts, P, u);
    const uint32_t r = u - cuts[x];
    for_each_run(indices, indptr[u], indptr[u + 1], cuts, [&](uint32_t y, uint32_t first, uint32_t cnt) {
      const uint32_t t = x * P + y;
      uint32_t* dst = col_pool + col_off[t] + rp_pool[rp_off[t] + r];
      const uint32_t base = cuts[y];
      for (uint32_t q = 0; q < cnt; q++) dst[q] = indices[first + q] - base;
    });
  }
}

__global__ void k_expand_rows(const uint32_t* __restrict__ indptr, uint32_t n, uint32_t* __restrict__ rows) {
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += stride)
    for (uint32_t e = indptr[u]; e < indptr[u + 1]; e++) rows[e] = u;
}

// rev_indptr[v] = first position of key v in the sorted keys (v in [0, n]).
__global__ void k_rev_indptr(const uint32_t* __restrict__ keys, uint64_t m, uint32_t n,
                             uint32_t* __restrict__ rev_indptr) {
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

struct DevBuf {
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() { return static_cast<T*>(p); }
};

int dalloc(DevBuf& b, size_t bytes) {
  cudaError_t e = cudaMalloc(&b.p, std::max<size_t>(bytes, 16));
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(BBTC_ERR_NOMEM, std::string("device allocation of ") + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
  }
  return BBTC_OK;
}

// Build one block CSR (forward or reversed) from a CSR in device memory.
int build_block(bbtc_ctx* ctx, BlockTiles& bt, const uint32_t* d_indptr, const uint32_t* d_indices, uint32_t n,
                uint64_t m, const std::vector<uint32_t>& cuts, const uint32_t* d_cuts, int grid) {
  const uint32_t P = (uint32_t)cuts.size() - 1;
  const uint32_t T = P * P;
  cudaStream_t s = ctx->stream;
  bt.P = P;
  bt.nnz.assign(T, 0);
  bt.maxdeg.assign(T, 0);
  bt.nerows.assign(T, 0);
  bt.rp_off.assign(T, kNoSegment);
  bt.col_off.assign(T, kNoSegment);

  DevBuf stats;
  BBTC_TRY(dalloc(stats, 3 * T * sizeof(uint32_t)));
  BBTC_CUDA(cudaMemsetAsync(stats.p, 0, 3 * T * sizeof(uint32_t), s));
  if (n > 0) {
    const size_t sm = (3 * T + P + 1) * sizeof(uint32_t);
    if (sm > 48 * 1024)
      BBTC_CUDA(cudaFuncSetAttribute(k_tile_count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_tile_count<<<grid, 256, sm, s>>>(d_indptr, d_indices, n, d_cuts, P, stats.as<uint32_t>(),
                                       stats.as<uint32_t>() + T, stats.as<uint32_t>() + 2 * T);
    BBTC_CUDA(cudaGetLastError());
  }
  std::vector<uint32_t> hst(3 * T);
  BBTC_CUDA(cudaMemcpyAsync(hst.data(), stats.p, 3 * T * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaStreamSynchronize(s));
  std::copy(hst.begin(), hst.begin() + T, bt.nnz.begin());
  std::copy(hst.begin() + T, hst.begin() + 2 * T, bt.maxdeg.begin());
  std::copy(hst.begin() + 2 * T, hst.end(), bt.nerows.begin());

  // segment offsets for the non-empty tiles, in row-major tile order
  std::vector<uint64_t> seg_start;
  std::vector<uint32_t> seg_base;
  uint64_t rp_cur = 0, col_cur = 0, nnz_cur = 0;
  for (uint32_t t = 0; t < T; t++) {
    if (!bt.nnz[t]) continue;
    const uint32_t x = t / P;
    const uint64_t H = (uint64_t)cuts[x + 1] - cuts[x];
    bt.rp_off[t] = rp_cur;
    bt.col_off[t] = col_cur;
    seg_start.push_back(rp_cur);
    seg_base.push_back((uint32_t)nnz_cur);
    rp_cur += align4(H + 1);
    col_cur += align4(bt.nnz[t]);
    nnz_cur += bt.nnz[t];
  }
  bt.rp_len = rp_cur + 4;  // a 16-byte tail keeps rounded-up bulk reads inside the pool
  bt.col_len = col_cur + 4;
  {
    cudaError_t e1 = cudaMalloc(&bt.d_rp, bt.rp_len * sizeof(uint32_t));
    cudaError_t e2 = cudaMalloc(&bt.d_col, bt.col_len * sizeof(uint32_t));
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
      cudaGetLastError();
      bt.release();
      return fail(BBTC_ERR_NOMEM, "device allocation of the block-CSR pools failed");
    }
  }
  if (seg_start.empty()) {
    BBTC_CUDA(cudaMemsetAsync(bt.d_rp, 0, bt.rp_len * sizeof(uint32_t), s));
    BBTC_CUDA(cudaMemsetAsync(bt.d_col, 0, bt.col_len * sizeof(uint32_t), s));
    return BBTC_OK;
  }
  DevBuf offs, segs, counts;
  BBTC_TRY(dalloc(offs, 2 * T * sizeof(uint64_t)));
  BBTC_TRY(dalloc(segs, seg_start.size() * (sizeof(uint64_t) + sizeof(uint32_t))));
  BBTC_TRY(dalloc(counts, bt.rp_len * sizeof(uint32_t)));
  uint64_t* d_rp_off = offs.as<uint64_t>();
  uint64_t* d_col_off = d_rp_off + T;
  uint64_t* d_seg_start = segs.as<uint64_t>();
  uint32_t* d_seg_base = reinterpret_cast<uint32_t*>(d_seg_start + seg_start.size());
  BBTC_CUDA(cudaMemcpyAsync(d_rp_off, bt.rp_off.data(), T * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  BBTC_CUDA(cudaMemcpyAsync(d_col_off, bt.col_off.data(), T * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
  BBTC_CUDA(cudaMemcpyAsync(d_seg_start, seg_start.data(), seg_start.size() * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, s));
  BBTC_CUDA(cudaMemcpyAsync(d_seg_base, seg_base.data(), seg_base.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s));
  BBTC_CUDA(cudaMemsetAsync(counts.p, 0, bt.rp_len * sizeof(uint32_t), s));
  BBTC_CUDA(cudaMemsetAsync(bt.d_col, 0, bt.col_len * sizeof(uint32_t), s));
  k_row_counts<<<grid, 256, 0, s>>>(d_indptr, d_indices, n, d_cuts, P, d_rp_off, counts.as<uint32_t>());
  BBTC_CUDA(cudaGetLastError());
  size_t tmp_bytes = 0;
  BBTC_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, counts.as<uint32_t>(), bt.d_rp,
                                          (int64_t)bt.rp_len, s));
  DevBuf tmp;
  BBTC_TRY(dalloc(tmp, tmp_bytes));
  BBTC_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmp_bytes, counts.as<uint32_t>(), bt.d_rp,
                                          (int64_t)bt.rp_len, s));
  k_localize<<<grid, 256, 0, s>>>(bt.d_rp, bt.rp_len, d_seg_start, d_seg_base, (uint32_t)seg_start.size());
  BBTC_CUDA(cudaGetLastError());
  k_scatter<<<grid, 256, 0, s>>>(d_indptr, d_indices, n, d_cuts, P, d_rp_off, d_col_off, bt.d_rp, bt.d_col);
  BBTC_CUDA(cudaGetLastError());
  BBTC_CUDA(cudaStreamSynchronize(s));  // the temporaries above are freed on return
  return BBTC_OK;
}

}  // namespace

void BlockTiles::release() {
  if (d_rp) cudaFree(d_rp);
  if (d_col) cudaFree(d_col);
  d_rp = d_col = nullptr;
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
  } else {
    d.rp = d.col = nullptr;
  }
  return d;
}

int build_layout(bbtc_graph* g, const uint32_t* d_indptr, const uint32_t* d_indices) {
  bbtc_ctx* ctx = g->ctx;
  cudaStream_t s = ctx->stream;
  const uint32_t n = g->n;
  const uint64_t m = g->m;
  const int grid = ctx->sms * 8;
  cudaEvent_t ev0, ev1;
  BBTC_CUDA(cudaEventCreate(&ev0));
  BBTC_CUDA(cudaEventCreate(&ev1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } evg{ev0, ev1};
  BBTC_CUDA(cudaEventRecord(ev0, s));

  DevBuf d_cuts, bad;
  BBTC_TRY(dalloc(d_cuts, g->cuts.size() * sizeof(uint32_t)));
  BBTC_TRY(dalloc(bad, sizeof(uint32_t)));
  BBTC_CUDA(cudaMemcpyAsync(d_cuts.p, g->cuts.data(), g->cuts.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
  BBTC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(uint32_t), s));
  if (n > 0) {
    k_validate<<<grid, 256, 0, s>>>(d_indptr, d_indices, n, m, bad.as<uint32_t>());
    BBTC_CUDA(cudaGetLastError());
  }
  uint32_t hbad = 0;
  BBTC_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaStreamSynchronize(s));
  if (hbad) {
    std::string why;
    if (hbad & 1) why += " indptr[0] != 0;";
    if (hbad & 2) why += " indptr[n] != m;";
    if (hbad & 4) why += " row pointers decrease or exceed m;";
    if (hbad & 8) why += " a column id >= n;";
    if (hbad & 16) why += " a row is not strictly increasing (unsorted or duplicate ids);";
    return fail(BBTC_ERR_INPUT, "CSR breaks the input contract:" + why);
  }

  BBTC_TRY(build_block(ctx, g->fwd, d_indptr, d_indices, n, m, g->cuts, d_cuts.as<uint32_t>(), grid));

  // reversed graph: stable sort of (column, row) pairs by column keeps each in-list sorted
  {
    DevBuf keys_in, keys_out, vals_in, vals_out, rev_indptr;
    BBTC_TRY(dalloc(keys_out, m * sizeof(uint32_t)));
    BBTC_TRY(dalloc(vals_in, m * sizeof(uint32_t)));
    BBTC_TRY(dalloc(vals_out, m * sizeof(uint32_t)));
    BBTC_TRY(dalloc(rev_indptr, ((size_t)n + 1) * sizeof(uint32_t)));
    if (m > 0) {
      k_expand_rows<<<grid, 256, 0, s>>>(d_indptr, n, vals_in.as<uint32_t>());
      BBTC_CUDA(cudaGetLastError());
      int end_bit = 1;
      while (end_bit < 32 && (1ull << end_bit) < (uint64_t)n) end_bit++;
      size_t tmp_bytes = 0;
      BBTC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_indices, keys_out.as<uint32_t>(),
                                                vals_in.as<uint32_t>(), vals_out.as<uint32_t>(), (int64_t)m,
                                                0, end_bit, s));
      DevBuf tmp;
      BBTC_TRY(dalloc(tmp, tmp_bytes));
      BBTC_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, d_indices, keys_out.as<uint32_t>(),
                                                vals_in.as<uint32_t>(), vals_out.as<uint32_t>(), (int64_t)m,
                                                0, end_bit, s));
      k_rev_indptr<<<grid, 256, 0, s>>>(keys_out.as<uint32_t>(), m, n, rev_indptr.as<uint32_t>());
      BBTC_CUDA(cudaGetLastError());
      BBTC_CUDA(cudaStreamSynchronize(s));
    } else {
      BBTC_CUDA(cudaMemsetAsync(rev_indptr.p, 0, ((size_t)n + 1) * sizeof(uint32_t), s));
    }
    BBTC_TRY(build_block(ctx, g->rev, rev_indptr.as<uint32_t>(), vals_out.as<uint32_t>(), n, m, g->cuts,
                         d_cuts.as<uint32_t>(), grid));
  }
  BBTC_CUDA(cudaEventRecord(ev1, s));
  BBTC_CUDA(cudaEventSynchronize(ev1));
  float ms = 0;
  BBTC_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  g->layout_ms = ms;
  g->device_bytes = (g->fwd.rp_len + g->fwd.col_len + g->rev.rp_len + g->rev.col_len) * sizeof(uint32_t) +
                    sizeof(uint64_t);
  return BBTC_OK;
}

}  // namespace bbtc

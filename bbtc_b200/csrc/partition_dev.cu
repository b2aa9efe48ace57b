// Cut vectors for a CSR that lives in device memory (the partitioner on the
// GPU): the same cuts as the host partitioners (partition.cpp) for the same
// CSR, without copying the CSR to the host.
//
// The reference computes its cuts on the host with the vendored SARMA
// library (include/utils/utils.hpp:271-288).
//
//  * uni: cuts[i] = i n / P.
//  * n1d: the smallest bottleneck B for which the greedy split of the row
//    pointer prefix into at most P stripes succeeds.  The host bisects over B
//    with one greedy probe per step; here one kernel evaluates 1024 candidate
//    bounds at once (a thread per bound, each a greedy probe over the device
//    row pointers), so four rounds narrow [max(maxrow, m/P), m] to the
//    minimum.  The cuts are the greedy probe at that minimum, as on the host.
//  * pal: the host draws the same sample of nonzero indices (a seeded
//    geometric-skip stream that needs only m), the GPU maps each sampled
//    index to its (row, column), and the probe runs on that sample on the
//    host (pal_from_sample).
#include <algorithm>
#include <cstring>
#include <vector>

#include "internal.h"
#include "partition_core.hpp"

namespace bbtc {
namespace {

constexpr uint32_t kCandidates = 1024;

__global__ void k_max_row(const uint32_t* __restrict__ indptr, uint32_t n, uint32_t* __restrict__ out) {
  uint32_t best = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    best = max(best, indptr[i + 1] - indptr[i]);
  best = __reduce_max_sync(0xffffffffu, best);
  if ((threadIdx.x & 31) == 0 && best) atomicMax(out, best);
}

// Greedy n1d probe for bound B (partition_core.hpp: n1d_probe): can the rows
// be split into at most P stripes of at most B nonzeros?
__device__ bool n1d_feasible(const uint32_t* __restrict__ indptr, uint32_t n, uint32_t P, uint64_t B) {
  uint32_t start = 0, k = 0;
  while (start < n) {
    if (k == P) return false;
    const uint64_t limit = (uint64_t)indptr[start] + B;
    // last index in [start, n] with indptr <= limit
    uint32_t lo = start, hi = n;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if ((uint64_t)indptr[mid] <= limit) lo = mid; else hi = mid - 1;
    }
    uint32_t end = lo;
    if (end <= start) end = start + 1;
    if ((uint64_t)indptr[end] - indptr[start] > B) return false;
    start = end;
    k++;
  }
  return true;
}

__global__ void k_n1d_candidates(const uint32_t* __restrict__ indptr, uint32_t n, uint32_t P, uint64_t lo,
                                 uint64_t step, uint64_t hi, uint8_t* __restrict__ ok) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= kCandidates) return;
  const uint64_t B = lo + (uint64_t)c * step;
  ok[c] = B <= hi ? (n1d_feasible(indptr, n, P, B) ? 1 : 0) : 2;  // 2: beyond the range
}

__global__ void k_n1d_cuts(const uint32_t* __restrict__ indptr, uint32_t n, uint32_t P, uint64_t B,
                           uint32_t* __restrict__ cuts) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t start = 0, k = 0;
  cuts[0] = 0;
  while (start < n && k < P) {
    const uint64_t limit = (uint64_t)indptr[start] + B;
    uint32_t lo = start, hi = n;
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if ((uint64_t)indptr[mid] <= limit) lo = mid; else hi = mid - 1;
    }
    uint32_t end = lo;
    if (end <= start) end = start + 1;
    start = end;
    k++;
    cuts[k] = start;
  }
  for (uint32_t t = k + 1; t <= P; t++) cuts[t] = n;
  cuts[P] = n;
}

// (row, column) of every sampled nonzero index.
__global__ void k_sample_rows(const uint64_t* __restrict__ edges, uint64_t M, const uint32_t* __restrict__ indptr,
                              uint32_t n, const uint32_t* __restrict__ indices, uint32_t* __restrict__ rows,
                              uint32_t* __restrict__ cols) {
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < M; t += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t e = edges[t];
    uint32_t lo = 0, hi = n;  // last r in [0, n] with indptr[r] <= e
    while (lo < hi) {
      const uint32_t mid = lo + (hi - lo + 1) / 2;
      if ((uint64_t)indptr[mid] <= e) lo = mid; else hi = mid - 1;
    }
    rows[t] = lo;
    cols[t] = indices[e];
  }
}

struct HostPinned {
  void* p = nullptr;
  ~HostPinned() {
    if (p) cudaFreeHost(p);
  }
};

int n1d_device(bbtc_ctx* ctx, uint32_t n, const uint32_t* d_indptr, uint64_t m, uint32_t P, uint32_t* cuts) {
  cudaStream_t s = ctx->stream;
  DevBuf dmax, ok, dcuts;
  BBTC_TRY(dalloc(dmax, sizeof(uint32_t), s));
  BBTC_TRY(dalloc(ok, kCandidates, s));
  BBTC_TRY(dalloc(dcuts, (P + 1) * sizeof(uint32_t), s));
  BBTC_CUDA(cudaMemsetAsync(dmax.p, 0, sizeof(uint32_t), s));
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(ctx->sms * 8, (n + 255) / 256));
  k_max_row<<<grid, 256, 0, s>>>(d_indptr, n, dmax.as<uint32_t>());
  BBTC_CUDA(cudaGetLastError());
  uint32_t* hmax = reinterpret_cast<uint32_t*>(ctx->h_stage + kStageBad);
  BBTC_CUDA(cudaMemcpyAsync(hmax, dmax.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaStreamSynchronize(s));
  // the host's search range (partition_core.hpp: n1d_cuts)
  uint64_t lo = std::max<uint64_t>(*hmax, (m + P - 1) / P);
  uint64_t hi = std::max<uint64_t>(m, lo);
  uint8_t* hok = reinterpret_cast<uint8_t*>(ctx->h_stage + kStageOut);
  while (lo < hi) {
    // hi is feasible; candidates lo, lo + step, ... cover [lo, hi]
    const uint64_t step = std::max<uint64_t>(1, (hi - lo + kCandidates) / kCandidates);
    k_n1d_candidates<<<kCandidates / 256, 256, 0, s>>>(d_indptr, n, P, lo, step, hi, ok.as<uint8_t>());
    BBTC_CUDA(cudaGetLastError());
    BBTC_CUDA(cudaMemcpyAsync(hok, ok.p, kCandidates, cudaMemcpyDeviceToHost, s));
    BBTC_CUDA(cudaStreamSynchronize(s));
    uint32_t first = kCandidates;
    for (uint32_t c = 0; c < kCandidates; c++)
      if (hok[c] == 1) {
        first = c;
        break;
      }
    if (first == kCandidates) {
      // every candidate below hi failed: the minimum lies above the last one
      uint32_t last = 0;
      for (uint32_t c = 0; c < kCandidates; c++)
        if (hok[c] == 0) last = c;
      lo = lo + (uint64_t)last * step + 1;
    } else {
      const uint64_t B = lo + (uint64_t)first * step;
      if (first > 0) lo = lo + (uint64_t)(first - 1) * step + 1;
      hi = B;
    }
  }
  k_n1d_cuts<<<1, 32, 0, s>>>(d_indptr, n, P, lo, dcuts.as<uint32_t>());
  BBTC_CUDA(cudaGetLastError());
  uint32_t* hc = reinterpret_cast<uint32_t*>(ctx->h_stage + kStageCuts);
  BBTC_CUDA(cudaMemcpyAsync(hc, dcuts.p, (P + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  BBTC_CUDA(cudaStreamSynchronize(s));
  std::memcpy(cuts, hc, (P + 1) * sizeof(uint32_t));
  return BBTC_OK;
}

int pal_device(bbtc_ctx* ctx, uint32_t n, const uint32_t* d_indptr, const uint32_t* d_indices, uint64_t m,
               uint32_t P, uint64_t seed, uint32_t* cuts) {
  cudaStream_t s = ctx->stream;
  const std::vector<uint64_t> es = pal_sample_edges(m, P, seed);
  const uint64_t M = es.size();
  std::vector<uint32_t> rows(M), cols(M);
  if (M) {
    HostPinned hp;
    BBTC_CUDA(cudaMallocHost(&hp.p, M * (sizeof(uint64_t) + 2 * sizeof(uint32_t))));
    uint64_t* he = static_cast<uint64_t*>(hp.p);
    uint32_t* hr = reinterpret_cast<uint32_t*>(he + M);
    uint32_t* hcol = hr + M;
    std::memcpy(he, es.data(), M * sizeof(uint64_t));
    DevBuf de, drc;
    BBTC_TRY(dalloc(de, M * sizeof(uint64_t), s));
    BBTC_TRY(dalloc(drc, 2 * M * sizeof(uint32_t), s));
    BBTC_CUDA(cudaMemcpyAsync(de.p, he, M * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)ctx->sms * 8, (M + 255) / 256));
    k_sample_rows<<<grid, 256, 0, s>>>(de.as<uint64_t>(), M, d_indptr, n, d_indices, drc.as<uint32_t>(),
                                       drc.as<uint32_t>() + M);
    BBTC_CUDA(cudaGetLastError());
    BBTC_CUDA(cudaMemcpyAsync(hr, drc.p, 2 * M * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    BBTC_CUDA(cudaStreamSynchronize(s));
    std::memcpy(rows.data(), hr, M * sizeof(uint32_t));
    std::memcpy(cols.data(), hcol, M * sizeof(uint32_t));
  }
  pal_from_sample(n, P, rows, cols, cuts);
  return BBTC_OK;
}

}  // namespace
}  // namespace bbtc

using namespace bbtc;

extern "C" int bbtc_cuts_device(bbtc_ctx* ctx, int kind, uint32_t n, const uint32_t* d_indptr,
                                const uint32_t* d_indices, uint64_t m, uint32_t P, uint64_t seed, uint32_t* cuts) {
  Range range("bbtc cuts");
  if (!ctx || !cuts) return fail(BBTC_ERR_ARG, "NULL argument");
  if (P < 1 || P > kMaxParts) return fail(BBTC_ERR_ARG, "P must be in [1, 64]");
  if (kind < 0 || kind > 2) return fail(BBTC_ERR_ARG, "kind must be 0 (uni), 1 (n1d) or 2 (pal)");
  if (kind != 0 && (!d_indptr || (m && !d_indices))) return fail(BBTC_ERR_ARG, "NULL CSR");
  if (m >= (1ull << 32)) return fail(BBTC_ERR_UNSUPPORTED, "m must be below 2^32 (32-bit row pointers)");
  if (n == 0) {
    for (uint32_t i = 0; i <= P; i++) cuts[i] = 0;
    return BBTC_OK;
  }
  if (kind == 0) {
    uniform_cuts(n, P, cuts);
    return BBTC_OK;
  }
  BBTC_CUDA(cudaSetDevice(ctx->device));
  if (kind == 1) return n1d_device(ctx, n, d_indptr, m, P, cuts);
  return pal_device(ctx, n, d_indptr, d_indices, m, P, seed, cuts);
}

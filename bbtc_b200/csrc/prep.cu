// Device-side input preparation.
//
// The reference prepares the counting graph on the host: it symmetrises the
// input, drops self-loops (include/utils/utils.hpp:172-250), relabels by
// ascending degree and keeps the upper triangle (SARMA csr_matrix.hpp:503-584).
// bbtc_orient_device does the same on the GPU with CUB sorts, for inputs that
// arrive as raw pairs in device memory; it also drops repeated pairs (the
// reference keeps repeated identical lines, PIGO csr.impl.hpp:51, which the
// counting contract here excludes).  Degree ties go by id, so the relabelling
// is a total order and the output equals the host pipeline's
// (bbtc_b200/csrc/graphgen.cpp) bit for bit.
//
// bbtc_rmat_device draws R-MAT pairs on the GPU with the host generator's
// counter-based stream (seed, pair index), so both generators give the same
// pairs for the same seed.
#include <cub/cub.cuh>

#include <algorithm>

#include "internal.h"

namespace bbtc {
namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// The host generator's stream: state = mix(seed * C ^ mix(index + D)), then
// successive splitmix64 outputs.
struct DevStream {
  uint64_t s;
  __device__ DevStream(uint64_t seed, uint64_t index)
      : s(mix64(seed * 0xD1B54A32D192ED03ull ^ mix64(index + 0x632BE59BD9B4E019ull))) {}
  __device__ __forceinline__ double uniform() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (z >> 11) * (1.0 / 9007199254740992.0);
  }
};

__global__ void k_rmat(int scale, uint64_t m, double a, double ab, double abc, uint64_t seed, uint32_t* __restrict__ src,
                       uint32_t* __restrict__ dst) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    DevStream rng(seed, e);
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
}

// (min, max) as one 64-bit key; self-loops and ids >= n become the largest key.
__global__ void k_canon(const uint32_t* __restrict__ src, const uint32_t* __restrict__ dst, uint64_t m, uint32_t n,
                        uint64_t* __restrict__ keys) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint32_t u = src[e], v = dst[e];
    keys[e] = (u == v || u >= n || v >= n) ? ~0ull : ((uint64_t)min(u, v) << 32) | max(u, v);
  }
}

__global__ void k_degrees(const uint64_t* __restrict__ keys, uint64_t m, uint32_t* __restrict__ deg) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint64_t k = keys[e];
    atomicAdd(&deg[k >> 32], 1u);
    atomicAdd(&deg[k & 0xffffffffull], 1u);
  }
}

__global__ void k_iota32(uint32_t* __restrict__ a, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] = i;
}

__global__ void k_rank(const uint32_t* __restrict__ order, uint32_t n, uint32_t* __restrict__ rank) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) rank[order[p]] = p;
}

// relabel both ends and orient from the lower to the higher new id
__global__ void k_relabel(const uint64_t* __restrict__ keys, uint64_t m, const uint32_t* __restrict__ rank,
                          uint64_t* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride) {
    const uint64_t k = keys[e];
    const uint32_t a = rank[k >> 32], b = rank[k & 0xffffffffull];
    out[e] = ((uint64_t)min(a, b) << 32) | max(a, b);
  }
}

__global__ void k_split(const uint64_t* __restrict__ keys, uint64_t m, uint32_t* __restrict__ indices) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += stride)
    indices[e] = (uint32_t)(keys[e] & 0xffffffffull);
}

// indptr[r] = first edge whose row is >= r
__global__ void k_indptr(const uint64_t* __restrict__ keys, uint64_t m, uint32_t n, uint32_t* __restrict__ indptr) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= n; r += gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
      const uint64_t mid = (lo + hi) >> 1;
      if ((keys[mid] >> 32) < r) lo = mid + 1; else hi = mid;
    }
    indptr[r] = (uint32_t)lo;
  }
}

int bits_for(uint64_t n) {
  int b = 1;
  while (b < 64 && (1ull << b) < n) b++;
  return b;
}

struct Buf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~Buf() {
    if (p) cudaFreeAsync(p, s);
  }
  template <class T>
  T* as() { return static_cast<T*>(p); }
};

int balloc(Buf& b, size_t bytes, cudaStream_t s) {
  b.s = s;
  if (dev_malloc(&b.p, std::max<size_t>(bytes, 16), s) != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(BBTC_ERR_NOMEM, "device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  return BBTC_OK;
}

}  // namespace
}  // namespace bbtc

using namespace bbtc;

extern "C" {

int bbtc_rmat_device(bbtc_ctx* ctx, int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                     uint32_t* d_src, uint32_t* d_dst) {
  if (!ctx || !d_src || !d_dst) return fail(BBTC_ERR_ARG, "NULL argument");
  if (scale < 1 || scale > 31 || edge_factor < 1) return fail(BBTC_ERR_ARG, "scale must be in [1, 31], edge factor >= 1");
  BBTC_CUDA(cudaSetDevice(ctx->device));
  const uint64_t m = (uint64_t)edge_factor << scale;
  k_rmat<<<ctx->sms * 8, 256, 0, ctx->stream>>>(scale, m, a, a + b, a + b + c, seed, d_src, d_dst);
  BBTC_CUDA(cudaGetLastError());
  BBTC_CUDA(cudaStreamSynchronize(ctx->stream));
  return BBTC_OK;
}

int bbtc_orient_device(bbtc_ctx* ctx, uint32_t n, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m_raw,
                       bbtc_csr_dev* out) {
  Range range("bbtc orient");
  if (!ctx || !out || (m_raw && (!d_src || !d_dst))) return fail(BBTC_ERR_ARG, "NULL argument");
  if (n == 0xffffffffu) return fail(BBTC_ERR_ARG, "n must be below 2^32 - 1");
  *out = bbtc_csr_dev{};
  BBTC_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const int grid = ctx->sms * 8;
  const int key_bits = 32 + bits_for(n);
  Buf keys, keys2, uniq, nsel, deg, ids, ids2, deg2, rank, tmp;
  BBTC_TRY(balloc(keys, std::max<uint64_t>(m_raw, 1) * 8, s));
  BBTC_TRY(balloc(keys2, std::max<uint64_t>(m_raw, 1) * 8, s));
  BBTC_TRY(balloc(nsel, 8, s));
  uint64_t m_und = 0;
  if (m_raw) {
    k_canon<<<grid, 256, 0, s>>>(d_src, d_dst, m_raw, n, keys.as<uint64_t>());
    BBTC_CUDA(cudaGetLastError());
    size_t tb = 0;
    BBTC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(), (int64_t)m_raw,
                                             0, 64, s));
    size_t tu = 0;
    BBTC_CUDA(cub::DeviceSelect::Unique(nullptr, tu, keys2.as<uint64_t>(), keys.as<uint64_t>(),
                                        nsel.as<uint64_t>(), (int64_t)m_raw, s));
    BBTC_TRY(balloc(tmp, std::max(tb, tu), s));
    BBTC_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, keys.as<uint64_t>(), keys2.as<uint64_t>(), (int64_t)m_raw, 0,
                                             64, s));
    BBTC_CUDA(cub::DeviceSelect::Unique(tmp.p, tu, keys2.as<uint64_t>(), keys.as<uint64_t>(), nsel.as<uint64_t>(),
                                        (int64_t)m_raw, s));
    uint64_t sel = 0, last = 0;
    BBTC_CUDA(cudaMemcpyAsync(&sel, nsel.p, 8, cudaMemcpyDeviceToHost, s));
    BBTC_CUDA(cudaStreamSynchronize(s));
    if (sel) {
      BBTC_CUDA(cudaMemcpyAsync(&last, keys.as<uint64_t>() + sel - 1, 8, cudaMemcpyDeviceToHost, s));
      BBTC_CUDA(cudaStreamSynchronize(s));
    }
    m_und = (sel && last == ~0ull) ? sel - 1 : sel;  // the dropped pairs sort last
  }
  if (m_und >= (1ull << 32)) return fail(BBTC_ERR_UNSUPPORTED, "more than 2^32 - 1 edges after cleaning");
  BBTC_TRY(balloc(deg, ((size_t)n + 1) * 4, s));
  BBTC_TRY(balloc(deg2, ((size_t)n + 1) * 4, s));
  BBTC_TRY(balloc(ids, ((size_t)n + 1) * 4, s));
  BBTC_TRY(balloc(ids2, ((size_t)n + 1) * 4, s));
  BBTC_TRY(balloc(rank, ((size_t)n + 1) * 4, s));
  BBTC_CUDA(cudaMemsetAsync(deg.p, 0, ((size_t)n + 1) * 4, s));
  if (m_und) {
    k_degrees<<<grid, 256, 0, s>>>(keys.as<uint64_t>(), m_und, deg.as<uint32_t>());
    BBTC_CUDA(cudaGetLastError());
  }
  if (n) {
    k_iota32<<<grid, 256, 0, s>>>(ids.as<uint32_t>(), n);
    BBTC_CUDA(cudaGetLastError());
    // stable sort of ids by degree: ties keep id order
    size_t tr = 0;
    BBTC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tr, deg.as<uint32_t>(), deg2.as<uint32_t>(), ids.as<uint32_t>(),
                                              ids2.as<uint32_t>(), (int64_t)n, 0, 32, s));
    Buf tmp2;
    BBTC_TRY(balloc(tmp2, tr, s));
    BBTC_CUDA(cub::DeviceRadixSort::SortPairs(tmp2.p, tr, deg.as<uint32_t>(), deg2.as<uint32_t>(), ids.as<uint32_t>(),
                                              ids2.as<uint32_t>(), (int64_t)n, 0, 32, s));
    k_rank<<<grid, 256, 0, s>>>(ids2.as<uint32_t>(), n, rank.as<uint32_t>());
    BBTC_CUDA(cudaGetLastError());
  }
  uint32_t* d_indptr = nullptr;
  uint32_t* d_indices = nullptr;
  if (dev_malloc(&d_indptr, ((size_t)n + 1) * 4, s) != cudaSuccess ||
      dev_malloc(&d_indices, std::max<uint64_t>(m_und, 1) * 4, s) != cudaSuccess) {
    cudaGetLastError();
    if (d_indptr) cudaFreeAsync(d_indptr, s);
    return fail(BBTC_ERR_NOMEM, "device allocation of the oriented CSR failed");
  }
  if (m_und) {
    k_relabel<<<grid, 256, 0, s>>>(keys.as<uint64_t>(), m_und, rank.as<uint32_t>(), keys2.as<uint64_t>());
    BBTC_CUDA(cudaGetLastError());
    size_t tb = 0;
    BBTC_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, keys2.as<uint64_t>(), keys.as<uint64_t>(), (int64_t)m_und, 0,
                                             key_bits, s));
    Buf tmp3;
    BBTC_TRY(balloc(tmp3, tb, s));
    BBTC_CUDA(cub::DeviceRadixSort::SortKeys(tmp3.p, tb, keys2.as<uint64_t>(), keys.as<uint64_t>(), (int64_t)m_und, 0,
                                             key_bits, s));
    k_split<<<grid, 256, 0, s>>>(keys.as<uint64_t>(), m_und, d_indices);
    BBTC_CUDA(cudaGetLastError());
  }
  k_indptr<<<grid, 256, 0, s>>>(keys.as<uint64_t>(), m_und, n, d_indptr);
  BBTC_CUDA(cudaGetLastError());
  BBTC_CUDA(cudaStreamSynchronize(s));
  out->indptr = d_indptr;
  out->indices = d_indices;
  out->n = n;
  out->m = m_und;
  return BBTC_OK;
}

int bbtc_csr_dev_free(bbtc_ctx* ctx, bbtc_csr_dev* csr) {
  if (!ctx || !csr) return fail(BBTC_ERR_ARG, "NULL argument");
  cudaSetDevice(ctx->device);
  if (csr->indptr) cudaFreeAsync(csr->indptr, ctx->stream);
  if (csr->indices) cudaFreeAsync(csr->indices, ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  *csr = bbtc_csr_dev{};
  return BBTC_OK;
}

}  // extern "C"

// Intersection kernels, the device work queue and the launch paths.
//
// A task (i, j, k) contributes sum_{r in part i} sum_{b in ab[r]} |ac[r] ∩ bc[b]|
// (the reference's SparseKernel / DenseKernel, src/triangle_counting/
// gpu_sparse_kernel.cu:6-49 and gpu_dense_kernel.cu:3-47, one thread per row
// of ab).  The same sum is taken here one *pivot row* at a time:
//
//   v-centric (default): for each row b of bc (vertex v of part j), the row
//     bc[b] becomes a membership structure in the warp's shared memory, and
//     every u with b in ab[u] -- the CSC column b of ab, i.e. the reversed
//     tile (j, i) -- streams its row ac[u] against it.  With the degree order
//     the ac rows are the shorter side, so this probes sum d_k(u) ids where the
//     reference's bitmap form probes sum d_k(v).
//   u-centric (the reference's row order): pivot = ac[r], the rows bc[b] for
//     b in ab[r] are streamed against it.
//
// Membership structures (TaskKind): a bitmap of the column part (when the part
// is at most 32 * bitmap_words ids wide), a sorted copy of the pivot row
// searched by bisection, or -- for pivot rows longer than the shared buffer --
// bisection in global memory.
//
// Work units are runs of `unit_edges` consecutive entries of the rows tile.
// In the persistent form every warp of a grid sized to the SM count claims
// units from one atomic head over all tasks (cost-sorted, heaviest first);
// in the plain form each task is one launch whose warps stride over its units.
// The per-probe-row work inside a unit is balanced across the 32 lanes with a
// merge-path split: the probe rows of 32 entries are concatenated and each lane
// takes one contiguous 1/32 of the ids.
#include <algorithm>
#include <cstring>
#include <sstream>

#include "internal.h"

namespace bbtc {

namespace {

constexpr uint32_t FULL = 0xffffffffu;
constexpr uint32_t kSegWords = 72;  // per-warp: 33 segment starts + 32 bases (+ pad)

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
  uint32_t first, last;
};

template <uint32_t KIND>
__device__ __forceinline__ uint32_t member(const uint32_t* bm, const PivotView& pv, uint32_t x) {
  if constexpr (KIND == kPivotBitmap) {
    return (bm[x >> 5] >> (x & 31)) & 1u;
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

// Probe the rows selected by entries [e, ee) of the rows tile against the
// pivot structure; returns this lane's hit count.
template <uint32_t KIND>
__device__ __forceinline__ uint32_t probe_entries(const uint32_t* __restrict__ rcol, uint32_t e, uint32_t ee,
                                                  const uint32_t* __restrict__ prb_rp,
                                                  const uint32_t* __restrict__ prb_col, const uint32_t* bm,
                                                  uint32_t* sstart, uint32_t* sbase, const PivotView& pv,
                                                  uint32_t lane) {
  uint32_t hits = 0;
  for (uint32_t base = e; base < ee; base += 32) {
    const uint32_t q = base + lane;
    uint32_t start = 0, len = 0;
    if (q < ee) {
      const uint32_t r = rcol[q];
      start = prb_rp[r];
      len = prb_rp[r + 1] - start;
    }
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
    sbase[lane] = start - excl;  // modular: sbase + p is the id's position for p in the segment
    if (lane == 31) sstart[32] = total;
    __syncwarp();
    const uint32_t per = (total + 31) >> 5;
    const uint32_t pbeg = lane * per;
    const uint32_t pend = min(pbeg + per, total);
    if (pbeg < pend) {
      uint32_t owner = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1)
        if (sstart[owner + step] <= pbeg) owner += step;
      uint32_t nb = sstart[owner + 1];
      uint32_t bs = sbase[owner];
      for (uint32_t p = pbeg; p < pend; p++) {
        while (p >= nb) {
          owner++;
          nb = sstart[owner + 1];
          bs = sbase[owner];
        }
        hits += member<KIND>(bm, pv, prb_col[bs + p]);
      }
    }
    __syncwarp();
  }
  return hits;
}

// One work unit: entries [unit*K, min((unit+1)*K, nnz)) of the rows tile.
template <uint32_t KIND>
__device__ __forceinline__ unsigned long long run_unit(const DevTask& tk, uint32_t unit, uint32_t* bm,
                                                       uint32_t* sstart, uint32_t* sbase, uint32_t lane) {
  const uint32_t* __restrict__ r_rp = tk.rows.rp;
  const uint32_t* __restrict__ r_col = tk.rows.col;
  const uint32_t* __restrict__ p_rp = tk.pivot.rp;
  const uint32_t* __restrict__ p_col = tk.pivot.col;
  const uint32_t* __restrict__ q_rp = tk.probe.rp;
  const uint32_t* __restrict__ q_col = tk.probe.col;
  const uint32_t H = tk.rows.H;
  const uint64_t e0 = (uint64_t)unit * tk.unit_edges;
  uint32_t e = (uint32_t)e0;
  const uint64_t e1w = e0 + tk.unit_edges;
  const uint32_t e1 = e1w < tk.rows.nnz ? (uint32_t)e1w : tk.rows.nnz;
  // row b holding entry e: the largest b with rp[b] <= e
  uint32_t b = 0;
  {
    uint32_t lo = 0, hi = H;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (r_rp[mid] <= e) lo = mid; else hi = mid;
    }
    b = lo;
  }
  unsigned long long acc = 0;
  while (e < e1) {
    const uint32_t ee = min(r_rp[b + 1], e1);
    const uint32_t ps = p_rp[b];
    const uint32_t pd = p_rp[b + 1] - ps;
    if (pd > 0) {
      const uint32_t* prow = p_col + ps;
      if constexpr (KIND == kPivotBitmap) {
        for (uint32_t i = lane; i < pd; i += 32) {
          const uint32_t x = prow[i];
          atomicOr(&bm[x >> 5], 1u << (x & 31));
        }
      } else if constexpr (KIND == kPivotList) {
        for (uint32_t i = lane; i < pd; i += 32) bm[i] = prow[i];
      }
      __syncwarp();
      PivotView pv;
      pv.row = prow;
      pv.len = pd;
      pv.first = prow[0];
      pv.last = prow[pd - 1];
      acc += probe_entries<KIND>(r_col, e, ee, q_rp, q_col, bm, sstart, sbase, pv, lane);
      if constexpr (KIND == kPivotBitmap) {
        if (pd < tk.words) {
          for (uint32_t i = lane; i < pd; i += 32) bm[prow[i] >> 5] = 0;
        } else {
          for (uint32_t i = lane; i < tk.words; i += 32) bm[i] = 0;
        }
      }
      __syncwarp();
    }
    e = ee;
    if (e < e1) {
      // next row with an entry at or after e
      b++;
      while (true) {
        const uint32_t idx = b + lane;
        const uint32_t v = idx < H ? r_rp[idx + 1] : 0xffffffffu;
        const uint32_t mask = __ballot_sync(FULL, v > e);
        if (mask) {
          b += __ffs(mask) - 1;
          break;
        }
        b += 32;
      }
    }
  }
  return acc;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(FULL, v, d);
  return v;
}

__device__ __forceinline__ unsigned long long dispatch_unit(const DevTask& tk, uint32_t unit, uint32_t* bm,
                                                            uint32_t* sstart, uint32_t* sbase, uint32_t lane) {
  switch (tk.kind) {
    case kPivotBitmap: return run_unit<kPivotBitmap>(tk, unit, bm, sstart, sbase, lane);
    case kPivotList: return run_unit<kPivotList>(tk, unit, bm, sstart, sbase, lane);
    default: return run_unit<kPivotGlobal>(tk, unit, bm, sstart, sbase, lane);
  }
}

// Persistent form: every warp claims units from one head until the queue is empty.
__global__ void __launch_bounds__(256) k_count_queue(const DevTask* __restrict__ tasks,
                                                     const uint32_t* __restrict__ prefix, uint32_t ntasks,
                                                     uint32_t total_units, uint32_t* __restrict__ head,
                                                     unsigned long long* __restrict__ outs, uint32_t bm_words) {
  extern __shared__ __align__(16) uint32_t sh[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* bm = sh + warp * (bm_words + kSegWords);
  uint32_t* sstart = bm + bm_words;
  uint32_t* sbase = sstart + 33;
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
    const DevTask& tk = tasks[lo];
    const unsigned long long c = warp_sum(dispatch_unit(tk, g - prefix[lo], bm, sstart, sbase, lane));
    if (lane == 0 && c) atomicAdd(&outs[tk.slot], c);
  }
}

// Plain form: one task per launch; warps stride over the task's units.
__global__ void __launch_bounds__(256) k_count_task(const DevTask* __restrict__ task, uint32_t units,
                                                    unsigned long long* __restrict__ outs, uint32_t bm_words) {
  extern __shared__ __align__(16) uint32_t sh[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* bm = sh + warp * (bm_words + kSegWords);
  uint32_t* sstart = bm + bm_words;
  uint32_t* sbase = sstart + 33;
  for (uint32_t i = lane; i < bm_words; i += 32) bm[i] = 0;
  __syncwarp();
  const DevTask& tk = *task;
  const uint32_t wpb = blockDim.x >> 5;
  unsigned long long acc = 0;
  for (uint32_t u = blockIdx.x * wpb + warp; u < units; u += gridDim.x * wpb)
    acc += dispatch_unit(tk, u, bm, sstart, sbase, lane);
  acc = warp_sum(acc);
  if (lane == 0 && acc) atomicAdd(&outs[tk.slot], acc);
}

size_t smem_bytes(uint32_t bm_words, uint32_t warps) {
  return (size_t)warps * (bm_words + kSegWords) * sizeof(uint32_t);
}

uint32_t norm_bm_words(uint32_t w) {
  if (w == 0) w = 2048;
  w = (w + 3) & ~3u;
  return std::max<uint32_t>(w, 32);
}

uint32_t norm_warps(uint32_t w) { return w == 0 ? 8 : std::min<uint32_t>(std::max<uint32_t>(w, 1), 8); }

}  // namespace

int kernel_smem_optin(bbtc_ctx* ctx, const bbtc_opts& o) {
  const size_t sm = smem_bytes(norm_bm_words(o.bitmap_words), norm_warps(o.warps_per_block));
  if (sm > ctx->smem_optin)
    return fail(BBTC_ERR_ARG, "bitmap_words x warps_per_block needs " + std::to_string(sm) +
                                  " bytes of shared memory; the device allows " + std::to_string(ctx->smem_optin));
  BBTC_CUDA(cudaFuncSetAttribute(k_count_queue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  BBTC_CUDA(cudaFuncSetAttribute(k_count_task, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  return BBTC_OK;
}

// Build the device task array for a request.  A single graph keeps the
// caller's task order (its border split); several graphs are merged into one
// queue ordered by estimated probe work, heaviest first.
static int make_plan(const std::vector<bbtc_graph*>& graphs, const std::vector<std::vector<bbtc_task>>& tasks,
                     const bbtc_opts& o, Plan* plan) {
  const uint32_t bmw = norm_bm_words(o.bitmap_words);
  const uint32_t unit_work = o.unit_work ? o.unit_work : 8192;
  std::vector<DevTask> list;
  std::vector<double> cost;
  for (size_t gi = 0; gi < graphs.size(); gi++) {
    const bbtc_graph* g = graphs[gi];
    const uint32_t P = g->P;
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
      const uint32_t W = d.pivot.W;
      d.words = (W + 31) / 32;
      const bool fits_bitmap = d.words <= bmw;
      const bool fits_list = d.pivot.maxdeg <= bmw;
      if (!u_centric && o.kernel != BBTC_KERNEL_SEARCH && fits_bitmap)
        d.kind = kPivotBitmap;
      else
        d.kind = fits_list ? kPivotList : kPivotGlobal;
      const uint32_t probe_tile = u_centric ? j * P + k : i * P + k;
      const uint32_t probe_rows = std::max<uint32_t>(1, g->fwd.nerows[probe_tile]);
      const double avg = std::max(1.0, (double)d.probe.nnz / probe_rows);
      uint32_t K = (uint32_t)std::min(16384.0, std::max(32.0, unit_work / avg));
      K = (K + 31) & ~31u;
      d.unit_edges = K;
      d.slot = (uint32_t)gi;
      list.push_back(d);
      cost.push_back((double)d.rows.nnz * avg);
    }
  }
  std::vector<uint32_t> order(list.size());
  for (uint32_t q = 0; q < order.size(); q++) order[q] = q;
  if (graphs.size() > 1)
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  plan->tasks.clear();
  plan->prefix.assign(1, 0);
  uint64_t total = 0;
  for (uint32_t q : order) {
    const DevTask& d = list[q];
    total += (d.rows.nnz + d.unit_edges - 1) / d.unit_edges;
    if (total >= 0xffffffffull) return fail(BBTC_ERR_UNSUPPORTED, "more than 2^32 work units in one request");
    plan->tasks.push_back(d);
    plan->prefix.push_back((uint32_t)total);
  }
  plan->total_units = (uint32_t)total;
  return BBTC_OK;
}

void Plan::release() {
  if (exec) cudaGraphExecDestroy(exec);
  if (d_tasks) cudaFree(d_tasks);
  if (d_prefix) cudaFree(d_prefix);
  exec = nullptr;
  d_tasks = nullptr;
  d_prefix = nullptr;
}

static int enqueue_launches(bbtc_ctx* ctx, Plan* plan, const bbtc_opts& o, uint64_t* d_outs, uint32_t nouts) {
  cudaStream_t s = ctx->stream;
  const uint32_t bmw = norm_bm_words(o.bitmap_words);
  const uint32_t wpb = norm_warps(o.warps_per_block);
  const size_t sm = smem_bytes(bmw, wpb);
  auto* outs = reinterpret_cast<unsigned long long*>(d_outs);
  BBTC_CUDA(cudaMemsetAsync(d_outs, 0, nouts * sizeof(uint64_t), s));
  plan->launches = 0;
  const uint32_t ntasks = (uint32_t)plan->tasks.size();
  if (ntasks == 0) return BBTC_OK;
  if (o.mode == BBTC_MODE_PLAIN) {
    for (uint32_t t = 0; t < ntasks; t++) {
      const uint32_t units = plan->prefix[t + 1] - plan->prefix[t];
      const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>((units + wpb - 1) / wpb, ctx->sms * 8));
      k_count_task<<<grid, wpb * 32, sm, s>>>(plan->d_tasks + t, units, outs, bmw);
      BBTC_CUDA(cudaGetLastError());
      plan->launches++;
    }
  } else {
    int per_sm = 0;
    BBTC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_count_queue, wpb * 32, sm));
    per_sm = std::max(1, per_sm);
    if (o.blocks_per_sm) per_sm = std::min<int>(per_sm, (int)o.blocks_per_sm);
    const uint32_t grid = ctx->sms * per_sm;
    BBTC_CUDA(cudaMemsetAsync(ctx->d_unit_counter, 0, sizeof(uint32_t), s));
    k_count_queue<<<grid, wpb * 32, sm, s>>>(plan->d_tasks, plan->d_prefix, ntasks, plan->total_units,
                                             ctx->d_unit_counter, outs, bmw);
    BBTC_CUDA(cudaGetLastError());
    plan->launches = 1;
  }
  return BBTC_OK;
}

int count_enqueue(bbtc_ctx* ctx, const std::vector<bbtc_graph*>& graphs,
                  const std::vector<std::vector<bbtc_task>>& tasks, const bbtc_opts& o, uint64_t* d_outs,
                  Plan* plan, bool reuse) {
  cudaStream_t s = ctx->stream;
  BBTC_TRY(kernel_smem_optin(ctx, o));
  if (!reuse) {
    plan->release();
    BBTC_TRY(make_plan(graphs, tasks, o, plan));
    const size_t nt = plan->tasks.size();
    if (nt) {
      if (cudaMalloc(&plan->d_tasks, nt * sizeof(DevTask)) != cudaSuccess ||
          cudaMalloc(&plan->d_prefix, (nt + 1) * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        plan->release();
        return fail(BBTC_ERR_NOMEM, "device allocation of the task queue failed");
      }
      BBTC_CUDA(cudaMemcpyAsync(plan->d_tasks, plan->tasks.data(), nt * sizeof(DevTask), cudaMemcpyHostToDevice, s));
      BBTC_CUDA(cudaMemcpyAsync(plan->d_prefix, plan->prefix.data(), (nt + 1) * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, s));
      BBTC_CUDA(cudaStreamSynchronize(s));  // host staging buffers must outlive the copies
    }
    plan->captured = false;
  }
  if (!o.use_cuda_graph) return enqueue_launches(ctx, plan, o, d_outs, (uint32_t)graphs.size());
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

}  // namespace bbtc

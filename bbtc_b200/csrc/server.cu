// Request server: continuous batching of count requests on one GPU.
//
// No counterpart in the reference (it counts one graph per process).  A
// request is a host CSR + cut vector; its answer is the exact count.
//
//   loader threads: take a pending request whose estimated device footprint
//     fits the HBM budget -- the smallest, or the oldest once it has waited
//     aging_ms -- build its device block CSR (upload + layout) on the
//     loader's stream for its size class (small: highest priority, a CSR in
//     page-locked host memory read by a kernel rather than the copy
//     engines; large: lowest priority, layout grids capped at 2 blocks per
//     SM, at most two 8 MiB upload pieces queued at a time), and queue it on its size
//     class's lane.  A request that could never fit fails with
//     BBTC_ERR_CAPACITY.  With two or more loaders half of them take small
//     requests only.
//   two launcher threads (lanes), each with its own highest-priority stream:
//     lane 0 counts graphs of at most small_edges edges, lane 1 the larger
//     ones with at most 3 blocks per SM, so a small request never waits for
//     a large count to drain the GPU.  A lane takes every ready graph of its
//     class (up to max_batch), counts them in one persistent launch with one
//     u64 slot per graph, publishes the counts, frees the graphs, returns
//     their memory to the budget.  The device memory pool is grown once at
//     creation.
//
// So requests that arrive while a launch is on the GPU are uploaded and laid
// out on the loader streams at the same time, and join the next launch; the
// device always holds the graphs being counted plus those being loaded.
// Every result is written to its own slot, so a graph's count does not depend
// on what shares its launch.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <new>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda.h>

#include "admission.hpp"
#include "internal.h"

namespace bbtc {

namespace {

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Device bytes a graph's layout needs, while it is built (upper bound).
uint64_t estimate_bytes(uint32_t n, uint64_t m, const std::vector<uint32_t>& cuts) {
  const uint64_t P = cuts.size() - 1;
  uint64_t rp = 0;
  for (uint64_t x = 0; x < P; x++) rp += P * (((uint64_t)cuts[x + 1] - cuts[x] + 1 + 3) & ~3ull);
  const uint64_t pools = 2 * 4 * (rp + 4) + 2 * 4 * (m + 4 * P * P + 4) + 8 * (m + 4 * P * P + 4) +
                        2 * 4 * (m / 32 + 2 * P * P + 2);
  const uint64_t csr = 4 * ((uint64_t)n + 1) + 4 * m;
  const uint64_t temps = 4 * (rp + 4) + 24 * m + 4 * ((uint64_t)n + 1) + (16ull << 20);
  return pools + csr + temps;
}

struct Request {
  uint64_t id = 0;
  uint32_t n = 0;
  uint64_t m = 0;
  const uint32_t* indptr = nullptr;
  const uint32_t* indices = nullptr;
  std::vector<uint32_t> cuts;
  uint64_t reserved = 0;  // bytes counted against the budget
  bbtc_graph* g = nullptr;
  int status = 0;  // 0 pending, 1 loading, 2 ready, 3 running, 4 done, < 0 failed
  uint64_t count = 0;
  uint32_t batch = 0;
  uint64_t t_submit = 0, t_done = 0, t_load = 0, t_ready = 0, t_launch = 0;
};

}  // namespace

void graph_release_on(bbtc_graph* g, cudaStream_t s);  // api.cu

}  // namespace bbtc

struct bbtc_server;

namespace bbtc {
namespace {

// One launch lane: a launcher thread with its own stream, result slots and
// ready queue.  Lane 0 counts the small graphs, lane 1 the large ones with
// its persistent grid capped per SM, so that lane 0's launches (and the
// loaders' layout kernels) always find room on every SM.
struct Lane {
  bbtc_ctx* ctx = nullptr;
  std::deque<Request*> ready;
  std::condition_variable cv;
  std::thread th;
  uint64_t* d_outs = nullptr;
  uint64_t* h_outs = nullptr;  // pinned: the readback waits only for this lane's stream
  uint32_t blocks_per_sm = 0;  // 0: as many as fit
  uint64_t launches = 0;
};

}  // namespace
}  // namespace bbtc

struct bbtc_server {
  bbtc_server_opts opts{};
  int device = 0;
  std::vector<bbtc_ctx*> load_ctx;  // two per loader: small requests, large requests
  std::mutex mu;
  std::condition_variable cv_load, cv_done;
  std::deque<bbtc::Request*> pending;
  bbtc::Lane lanes[2];
  std::unordered_map<uint64_t, bbtc::Request*> all;
  uint64_t next_id = 1;
  uint64_t in_use = 0;
  uint32_t loading = 0;
  uint32_t loading_large = 0;  // large requests being uploaded / laid out
  bool stop = false;
  std::vector<std::thread> loaders;
  CUgreenCtx green[2] = {nullptr, nullptr};  // SM partitions (small_sms > 0): small requests, large requests
  uint32_t green_sms[2] = {0, 0};
  // statistics
  uint64_t counted = 0, max_batch_seen = 0;
};

namespace bbtc {
namespace {

constexpr size_t kPickScan = 4096;  // pending requests a loader looks at per pick

uint32_t lane_of(const bbtc_server* s, const Request* r) { return r->m <= s->opts.small_edges ? 0u : 1u; }

// The next request a loader takes (admission.hpp), removed from `pending`, or nullptr.
Request* pick(bbtc_server* s, bool small_only) {
  AdmitLimits lim{s->opts.hbm_budget, s->in_use, s->opts.small_edges,
                  (uint64_t)s->opts.aging_ms * 1000000ull, now_ns(), small_only, kPickScan};
  lim.large_ok = !s->opts.max_large_loads || s->loading_large < s->opts.max_large_loads;
  lim.small_aging_ns = (uint64_t)s->opts.small_aging_us * 1000ull;
  const size_t best = admit_pick(s->pending, lim);
  if (best == SIZE_MAX) return nullptr;
  Request* r = s->pending[best];
  s->pending.erase(s->pending.begin() + (std::ptrdiff_t)best);
  return r;
}

void loader_main(bbtc_server* s, bbtc_ctx* ctx_small, bbtc_ctx* ctx_large, bool small_only) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    Request* r = nullptr;
    s->cv_load.wait(lk, [&] { return s->stop || (r = pick(s, small_only)) != nullptr; });
    if (s->stop) {
      if (r) s->pending.push_front(r);
      return;
    }
    if (r->reserved > s->opts.hbm_budget) {  // can never fit
      r->status = BBTC_ERR_CAPACITY;
      r->t_done = now_ns();
      s->cv_done.notify_all();
      continue;
    }
    s->in_use += r->reserved;
    r->status = 1;
    r->t_load = now_ns();
    s->loading++;
    const bool large = lane_of(s, r) == 1;
    if (large) s->loading_large++;
    lk.unlock();
    bbtc_graph* g = nullptr;
    // a large layout runs on a low-priority stream with its grids capped, so
    // the small ones' kernels are scheduled first and find free SMs
    bbtc_ctx* ctx = lane_of(s, r) == 0 ? ctx_small : ctx_large;
    const int rc = bbtc_graph_upload(ctx, r->n, r->indptr, r->indices, r->m, r->cuts.data(),
                                     (uint32_t)r->cuts.size() - 1, &g);
    lk.lock();
    s->loading--;
    if (large) s->loading_large--;
    if (rc != BBTC_OK) {
      s->in_use -= r->reserved;
      r->reserved = 0;
      r->status = rc;
      r->t_done = now_ns();
      s->cv_done.notify_all();
      s->cv_load.notify_all();
      continue;
    }
    // the layout is built: hold its real size
    s->in_use = s->in_use - r->reserved + g->device_bytes;
    r->reserved = g->device_bytes;
    r->g = g;
    r->status = 2;
    r->t_ready = now_ns();
    Lane& L = s->lanes[lane_of(s, r)];
    L.ready.push_back(r);
    L.cv.notify_one();
    s->cv_load.notify_all();
  }
}

void launcher_main(bbtc_server* s, uint32_t lane) {
  cudaSetDevice(s->device);
  Lane& L = s->lanes[lane];
  bbtc_ctx* ctx = L.ctx;
  std::unique_lock<std::mutex> lk(s->mu);
  Plan plan;
  while (true) {
    L.cv.wait(lk, [&] { return s->stop || !L.ready.empty(); });
    if (s->stop && L.ready.empty()) break;
    std::vector<Request*> batch;
    while (!L.ready.empty() && batch.size() < s->opts.max_batch) {
      batch.push_back(L.ready.front());
      L.ready.pop_front();
    }
    const uint64_t t_launch = now_ns();
    for (Request* r : batch) {
      r->status = 3;
      r->t_launch = t_launch;
    }
    lk.unlock();
    std::vector<bbtc_graph*> gs;
    std::vector<std::vector<bbtc_task>> tl(batch.size());
    for (Request* r : batch) gs.push_back(r->g);
    bbtc_opts o = s->opts.count;
    o.use_cuda_graph = 0;
    if (L.blocks_per_sm && (!o.blocks_per_sm || o.blocks_per_sm > L.blocks_per_sm)) o.blocks_per_sm = L.blocks_per_sm;
    const bool fused = o.kernel == BBTC_KERNEL_FUSED || (o.kernel == BBTC_KERNEL_AUTO && o.mode == BBTC_MODE_PERSISTENT);
    int rc = BBTC_OK;
    if (!fused) {
      for (size_t i = 0; i < batch.size(); i++) {
        if (rc == BBTC_OK) rc = ensure_fwd(gs[i]);
        uint32_t nt = 0;
        bbtc_task_list(gs[i]->P, nullptr, 0, &nt);
        tl[i].resize(nt);
        bbtc_task_list(gs[i]->P, tl[i].data(), nt, &nt);
      }
    }
    if (rc == BBTC_OK) rc = count_enqueue(ctx, gs, tl, o, fused, L.d_outs, &plan, false);
    if (rc == BBTC_OK) {
      const cudaError_t e =
          cudaMemcpyAsync(L.h_outs, L.d_outs, batch.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                          ctx->stream);
      const cudaError_t e2 = e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
      if (e2 != cudaSuccess) rc = cuda_fail(e2, "server batch readback");
      else rc = staging_status(ctx);
    }
    const uint64_t t = now_ns();
    // stream-ordered frees: the memory returns to the pool behind this launch
    for (Request* r : batch) graph_release_on(r->g, ctx->stream);
    lk.lock();
    for (size_t i = 0; i < batch.size(); i++) {
      Request* r = batch[i];
      r->g = nullptr;
      s->in_use -= r->reserved;
      r->reserved = 0;
      r->batch = (uint32_t)batch.size();
      r->t_done = t;
      if (rc == BBTC_OK) {
        r->count = L.h_outs[i];
        r->status = 4;
      } else {
        r->status = rc;
      }
    }
    L.launches++;
    s->counted += batch.size();
    s->max_batch_seen = std::max<uint64_t>(s->max_batch_seen, batch.size());
    s->cv_done.notify_all();
    s->cv_load.notify_all();
  }
  lk.unlock();
  plan.release();
}

// The driver's green-context calls (SM partitions), looked up once at the
// version this library was built with; `ok` is false when the driver lacks
// any of them.
struct GreenApi {
  CUresult (*get_device)(CUdevice*, int) = nullptr;
  CUresult (*get_resource)(CUdevice, CUdevResource*, CUdevResourceType) = nullptr;
  CUresult (*split)(CUdevResource*, unsigned*, const CUdevResource*, CUdevResource*, unsigned, unsigned) = nullptr;
  CUresult (*gen_desc)(CUdevResourceDesc*, CUdevResource*, unsigned) = nullptr;
  CUresult (*create)(CUgreenCtx*, CUdevResourceDesc, CUdevice, unsigned) = nullptr;
  CUresult (*stream)(CUstream*, CUgreenCtx, unsigned, int) = nullptr;
  CUresult (*destroy)(CUgreenCtx) = nullptr;
  bool ok = false;
};

const GreenApi& green_api() {
  static const GreenApi api = [] {
    GreenApi a;
    auto get = [](const char* name, void* fn) {
      cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
      const bool found = cudaGetDriverEntryPointByVersion(name, static_cast<void**>(fn), CUDA_VERSION,
                                                          cudaEnableDefault, &q) == cudaSuccess &&
                         q == cudaDriverEntryPointSuccess;
      cudaGetLastError();
      return found;
    };
    a.ok = get("cuDeviceGet", &a.get_device) && get("cuDeviceGetDevResource", &a.get_resource) &&
           get("cuDevSmResourceSplitByCount", &a.split) && get("cuDevResourceGenerateDesc", &a.gen_desc) &&
           get("cuGreenCtxCreate", &a.create) && get("cuGreenCtxStreamCreate", &a.stream) &&
           get("cuGreenCtxDestroy", &a.destroy);
    return a;
  }();
  return api;
}

// Split the device's SMs into two green contexts: `small_sms` (rounded up by
// the driver to its granularity, 8 on this architecture) for the small
// requests, the rest for the large ones.  Kernels launched into a stream of
// either run only on its SMs.
int make_partitions(bbtc_server* s, uint32_t small_sms) {
  const GreenApi& g = green_api();
  if (!g.ok) return fail(BBTC_ERR_UNSUPPORTED, "the driver offers no green contexts (SM partitions)");
  CUdevice dev = 0;
  CUdevResource all{}, part{}, rest{};
  unsigned groups = 1;
  if (g.get_device(&dev, s->device) != CUDA_SUCCESS ||
      g.get_resource(dev, &all, CU_DEV_RESOURCE_TYPE_SM) != CUDA_SUCCESS)
    return fail(BBTC_ERR_CUDA, "reading the device's SM resource failed");
  if (small_sms >= all.sm.smCount)
    return fail(BBTC_ERR_ARG, "small_sms must leave SMs for the large requests");
  if (g.split(&part, &groups, &all, &rest, 0, small_sms) != CUDA_SUCCESS || groups != 1 || rest.sm.smCount == 0)
    return fail(BBTC_ERR_ARG, "the SMs could not be split into the requested partition");
  CUdevResourceDesc d0 = nullptr, d1 = nullptr;
  if (g.gen_desc(&d0, &part, 1) != CUDA_SUCCESS || g.gen_desc(&d1, &rest, 1) != CUDA_SUCCESS ||
      g.create(&s->green[0], d0, dev, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS ||
      g.create(&s->green[1], d1, dev, CU_GREEN_CTX_DEFAULT_STREAM) != CUDA_SUCCESS)
    return fail(BBTC_ERR_CUDA, "creating the green contexts failed");
  s->green_sms[0] = part.sm.smCount;
  s->green_sms[1] = rest.sm.smCount;
  return BBTC_OK;
}

// Move a context onto a stream of SM partition `p` (its grids are then sized to the partition's SMs).
int set_partition_stream(bbtc_server* s, bbtc_ctx* c, int p, int priority) {
  CUstream st = nullptr;
  if (green_api().stream(&st, s->green[p], CU_STREAM_NON_BLOCKING, priority) != CUDA_SUCCESS)
    return fail(BBTC_ERR_CUDA, "creating a stream in an SM partition failed");
  cudaStreamDestroy(c->stream);
  c->stream = reinterpret_cast<cudaStream_t>(st);
  c->sms = (int)s->green_sms[p];
  return BBTC_OK;
}

// Give a context's stream the requested priority (lower numbers run first).
int set_stream_priority(bbtc_ctx* c, int priority) {
  cudaStream_t st = nullptr;
  BBTC_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, priority));
  cudaStreamDestroy(c->stream);
  c->stream = st;
  return BBTC_OK;
}

void fill_info(const Request* r, bbtc_request_info* info) {
  info->count = r->count;
  info->status = r->status == 4 ? 1 : (r->status < 0 ? r->status : 0);
  info->batch = r->batch;
  info->submit_ns = r->t_submit;
  info->done_ns = r->t_done;
  info->load_ns = r->t_load;
  info->ready_ns = r->t_ready;
  info->launch_ns = r->t_launch;
}

}  // namespace
}  // namespace bbtc

using namespace bbtc;

extern "C" {

void bbtc_server_opts_default(bbtc_server_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->hbm_budget = 150ull << 30;
  o->max_batch = 4096;
  o->max_requests = 1u << 20;
  // six loaders, at most two of them on large requests at a time: small
  // requests seldom wait for a loader (R-MAT s12-s22 mix at 1,208 req/s:
  // scale <= 18 p99 5.0 ms, against 5.6 ms with four loaders and no limit)
  o->loaders = 6;
  o->max_large_loads = 2;
  bbtc_opts_default(&o->count);
  o->small_edges = 1ull << 22;
  o->large_blocks_per_sm = 0;
  o->aging_ms = 50;
  o->pool_bytes = 0;
}

int bbtc_server_create(int device, const bbtc_server_opts* opts, bbtc_server** out) {
  if (!out) return fail(BBTC_ERR_ARG, "out is NULL");
  // one hardware work queue per stream: with the default 8, a small lane's
  // launch that hashed onto the large lane's queue waited for its count to
  // finish.  Takes effect only if CUDA is not initialised in the process yet.
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
  *out = nullptr;
  bbtc_server* s = new (std::nothrow) bbtc_server();
  if (!s) return fail(BBTC_ERR_NOMEM, "host allocation failed");
  if (opts) s->opts = *opts; else bbtc_server_opts_default(&s->opts);
  if (!s->opts.hbm_budget) s->opts.hbm_budget = 150ull << 30;
  if (!s->opts.max_batch) s->opts.max_batch = 4096;
  if (!s->opts.max_requests) s->opts.max_requests = 1u << 20;
  if (!s->opts.loaders) s->opts.loaders = 6;
  s->opts.loaders = std::min<uint32_t>(s->opts.loaders, 16);
  if (!s->opts.small_edges) s->opts.small_edges = 1ull << 22;
  s->device = device;
  int lo = 0, hi = 0;
  int rc = BBTC_OK;
  if (cudaSetDevice(device) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&lo, &hi) != cudaSuccess) {
    cudaGetLastError();
    lo = hi = 0;
  }
  // Stream priorities: both lanes and the small requests' loads highest, the
  // large requests' loads lowest (lower numbers run first).
  const int mid = hi;
  for (uint32_t l = 0; rc == BBTC_OK && l < 2; l++) {
    rc = bbtc_ctx_create(device, &s->lanes[l].ctx);
    if (rc == BBTC_OK) rc = set_stream_priority(s->lanes[l].ctx, hi);
  }
  for (uint32_t i = 0; rc == BBTC_OK && i < 2 * s->opts.loaders; i++) {
    bbtc_ctx* c = nullptr;
    rc = bbtc_ctx_create(device, &c);
    if (rc == BBTC_OK) s->load_ctx.push_back(c);
    if (rc == BBTC_OK) rc = set_stream_priority(c, i % 2 == 0 ? mid : lo);
    if (rc == BBTC_OK && i % 2 == 1) {
      c->layout_blocks_per_sm = s->opts.large_layout_blocks_per_sm ? s->opts.large_layout_blocks_per_sm : 2;
      c->upload_window = 2;
      // a large layout's passes hold SMs for milliseconds: with the largest
      // shared-memory carveout a small request's CUB passes and counts can
      // start beside them (small-request load p99 with an R-MAT s22 request in
      // flight: 2.1 ms -> 0.58 ms)
      c->open_carveout = true;
    }
    // small requests from page-locked buffers are read by a kernel: their
    // copies otherwise waited behind large uploads on the copy engines
    // (p99 4.1 ms for a copy whose median is 0.03 ms)
    if (rc == BBTC_OK && i % 2 == 0 && !s->opts.copy_engine_uploads)
      c->zero_copy_bytes = 4 * std::max<uint64_t>(s->opts.small_edges, 1ull << 22) + 64;
  }
  if (rc == BBTC_OK && s->opts.small_sms) {
    // lane 0 and every loader's small-request context on the small
    // partition, lane 1 and the large-request contexts on the other
    rc = make_partitions(s, s->opts.small_sms);
    for (uint32_t l = 0; rc == BBTC_OK && l < 2; l++) rc = set_partition_stream(s, s->lanes[l].ctx, (int)l, hi);
    for (uint32_t i = 0; rc == BBTC_OK && i < s->load_ctx.size(); i++)
      rc = set_partition_stream(s, s->load_ctx[i], (int)(i % 2), i % 2 == 0 ? mid : lo);
  }
  for (uint32_t l = 0; rc == BBTC_OK && l < 2; l++) {
    if (dev_malloc_sync(&s->lanes[l].d_outs, s->opts.max_batch * sizeof(uint64_t)) != cudaSuccess ||
        cudaMallocHost(&s->lanes[l].h_outs, s->opts.max_batch * sizeof(uint64_t)) != cudaSuccess) {
      cudaGetLastError();
      rc = fail(BBTC_ERR_NOMEM, "allocation of the result slots failed");
    }
  }
  if (rc != BBTC_OK) {
    for (auto* c : s->load_ctx) bbtc_ctx_destroy(c);
    for (auto& L : s->lanes) {
      if (L.ctx) bbtc_ctx_destroy(L.ctx);
      if (L.d_outs) cudaFree(L.d_outs);
      if (L.h_outs) cudaFreeHost(L.h_outs);
    }
    for (CUgreenCtx g : s->green)
      if (g) green_api().destroy(g);
    delete s;
    return rc;
  }
  {
    // the large lane uses at most 3 blocks per SM, so every SM keeps room
    // for the small lane's blocks
    s->lanes[1].blocks_per_sm = s->opts.large_blocks_per_sm ? s->opts.large_blocks_per_sm : 3;
  }
  {
    // memory freed on one stream is handed to another only once the free has
    // completed: with reuse that follows event dependencies, a small load
    // whose allocation took blocks a large load had just freed waited behind
    // that load (and the counts ahead of it) for tens of milliseconds
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      int off = 0;
      cudaMemPoolSetAttribute(pool, cudaMemPoolReuseFollowEventDependencies, &off);
      cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &off);
    }
    cudaGetLastError();
  }
  {
    // grow the device's memory pool once, now, to what the admission budget
    // can hold: a pool that grows while loads and counts run stalled every
    // loader for hundreds of milliseconds (up to 1.5 s when it grew by GBs)
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      cudaGetLastError();
      free_b = 0;
    }
    const uint64_t cap = free_b > (8ull << 30) ? free_b - (8ull << 30) : free_b / 2;
    const uint64_t want =
        std::min<uint64_t>(s->opts.pool_bytes ? s->opts.pool_bytes : s->opts.hbm_budget + s->opts.hbm_budget / 10, cap);
    cudaStream_t st = s->lanes[0].ctx->stream;
    void* p = nullptr;
    if (cudaMallocAsync(&p, want, st) == cudaSuccess) {
      cudaFreeAsync(p, st);
      cudaStreamSynchronize(st);
    } else {
      cudaGetLastError();  // not fatal: the pool grows on demand instead
    }
  }
  // with two or more loaders, half of them (rounded down) take small requests only
  const uint32_t small_only = s->opts.loaders > 1 ? s->opts.loaders / 2 : 0;
  for (size_t i = 0; i < s->opts.loaders; i++)
    s->loaders.emplace_back(loader_main, s, s->load_ctx[2 * i], s->load_ctx[2 * i + 1], i < small_only);
  for (uint32_t l = 0; l < 2; l++) s->lanes[l].th = std::thread(launcher_main, s, l);
  *out = s;
  return BBTC_OK;
}

int bbtc_server_destroy(bbtc_server* s) {
  if (!s) return BBTC_OK;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    // requests not yet loading fail; loads in progress and ready graphs finish first
    for (Request* r : s->pending) {
      r->status = BBTC_ERR_STATE;
      r->t_done = now_ns();
    }
    s->pending.clear();
    s->cv_done.wait(lk, [&] { return s->loading == 0; });
    s->stop = true;
    s->cv_load.notify_all();
    for (auto& L : s->lanes) L.cv.notify_all();
  }
  for (auto& t : s->loaders) t.join();
  for (auto& L : s->lanes) L.th.join();
  for (auto& kv : s->all) {
    if (kv.second->g) graph_release_on(kv.second->g, s->lanes[0].ctx->stream);
    delete kv.second;
  }
  cudaSetDevice(s->device);
  for (auto& L : s->lanes) {
    cudaStreamSynchronize(L.ctx->stream);
    cudaFree(L.d_outs);
    cudaFreeHost(L.h_outs);
  }
  for (auto* c : s->load_ctx) bbtc_ctx_destroy(c);
  for (auto& L : s->lanes) bbtc_ctx_destroy(L.ctx);
  for (CUgreenCtx g : s->green)  // after the streams in them are destroyed
    if (g) green_api().destroy(g);
  {
    // hand the pool's unused memory back (it was grown to the budget at creation)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
  }
  delete s;
  return BBTC_OK;
}

int bbtc_submit(bbtc_server* s, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m,
                const uint32_t* cuts, uint32_t P, uint64_t* req_id) {
  if (!s || !indptr || (m && !indices) || !cuts || !req_id) return fail(BBTC_ERR_ARG, "NULL argument");
  if (P < 1 || P > kMaxParts) return fail(BBTC_ERR_ARG, "P must be in [1, 64]");
  Request* r = new (std::nothrow) Request();
  if (!r) return fail(BBTC_ERR_NOMEM, "host allocation failed");
  r->n = n;
  r->m = m;
  r->indptr = indptr;
  r->indices = indices;
  r->cuts.assign(cuts, cuts + P + 1);
  r->reserved = estimate_bytes(n, m, r->cuts);
  r->t_submit = now_ns();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) {
    delete r;
    return fail(BBTC_ERR_STATE, "server is shutting down");
  }
  if (s->all.size() >= s->opts.max_requests) {
    delete r;
    return fail(BBTC_ERR_CAPACITY, "too many requests held; release finished ones with bbtc_release");
  }
  r->id = s->next_id++;
  s->all[r->id] = r;
  s->pending.push_back(r);
  *req_id = r->id;
  s->cv_load.notify_all();  // a loader reserved for small requests may not take this one
  return BBTC_OK;
}

int bbtc_poll(bbtc_server* s, uint64_t req_id, bbtc_request_info* info) {
  if (!s || !info) return fail(BBTC_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(req_id);
  if (it == s->all.end()) return fail(BBTC_ERR_STATE, "unknown request id");
  fill_info(it->second, info);
  return BBTC_OK;
}

int bbtc_wait(bbtc_server* s, uint64_t req_id, int64_t timeout_ms, bbtc_request_info* info) {
  if (!s || !info) return fail(BBTC_ERR_ARG, "NULL argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(req_id);
  if (it == s->all.end()) return fail(BBTC_ERR_STATE, "unknown request id");
  Request* r = it->second;
  auto finished = [&] { return r->status == 4 || r->status < 0; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, finished);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), finished)) {
    fill_info(r, info);
    return fail(BBTC_ERR_TIMEOUT, "request not finished within the timeout");
  }
  fill_info(r, info);
  return BBTC_OK;
}

int bbtc_release(bbtc_server* s, uint64_t req_id) {
  if (!s) return fail(BBTC_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(req_id);
  if (it == s->all.end()) return fail(BBTC_ERR_STATE, "unknown request id");
  Request* r = it->second;
  if (!(r->status == 4 || r->status < 0)) return fail(BBTC_ERR_STATE, "request still in flight");
  delete r;
  s->all.erase(it);
  return BBTC_OK;
}

int bbtc_server_stats_get(bbtc_server* s, bbtc_server_stats* st) {
  if (!s || !st) return fail(BBTC_ERR_ARG, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  st->launches = s->lanes[0].launches + s->lanes[1].launches;
  st->counted = s->counted;
  st->max_batch = s->max_batch_seen;
  st->pending = s->pending.size();
  st->ready = s->lanes[0].ready.size() + s->lanes[1].ready.size();
  st->device_bytes_in_use = s->in_use;
  return BBTC_OK;
}

}  // extern "C"

// C ABI of libbbtc.so: contexts, graphs, task lists and counting.
// The mapping to the reference's classes is given in include/bbtc_gpu.h.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <numeric>
#include <sstream>

#include "internal.h"

namespace bbtc {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int status, const std::string& msg) {
  set_error(msg);
  return status;
}

// Armed allocation fault: k >= 0 lets k more device allocations pass and fails
// the next one; -1 is disarmed.
static std::atomic<int64_t> g_alloc_fault{[] {
  const char* v = std::getenv("BBTC_FAIL_ALLOC");
  if (!v || !*v) return (int64_t)-1;
  char* end = nullptr;
  const long long k = std::strtoll(v, &end, 10);
  return *end == '\0' && k >= 0 ? (int64_t)k : (int64_t)-1;  // anything but a count leaves it disarmed
}()};

bool take_alloc_fault() {
  int64_t v = g_alloc_fault.load(std::memory_order_relaxed);
  while (v >= 0)
    if (g_alloc_fault.compare_exchange_weak(v, v - 1, std::memory_order_relaxed)) return v == 0;
  return false;
}

int cuda_fail(cudaError_t e, const char* what) {
  std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();  // clear a non-sticky error
  if (e == cudaErrorMemoryAllocation) return fail(BBTC_ERR_NOMEM, msg);
  if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice || e == cudaErrorInsufficientDriver)
    return fail(BBTC_ERR_NODEV, msg);
  return fail(BBTC_ERR_CUDA, msg);
}

namespace {

int validate_cuts(uint32_t n, const uint32_t* cuts, uint32_t P) {
  if (!cuts) return fail(BBTC_ERR_ARG, "cuts is NULL");
  if (P < 1 || P > kMaxParts) return fail(BBTC_ERR_ARG, "P must be in [1, 64]");
  if (cuts[0] != 0) return fail(BBTC_ERR_INPUT, "cuts[0] must be 0");
  for (uint32_t i = 0; i < P; i++)
    if (cuts[i + 1] < cuts[i]) return fail(BBTC_ERR_INPUT, "cuts must be non-decreasing");
  if (cuts[P] < n) return fail(BBTC_ERR_INPUT, "cuts[P] must be >= n");
  return BBTC_OK;
}

std::string plan_key(const std::vector<bbtc_graph*>& graphs, const std::vector<std::vector<bbtc_task>>& tasks,
                     const bbtc_opts& o) {
  // FNV-1a over the request: graphs, tasks and every option that shapes the launch
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](const void* p, size_t n) {
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) h = (h ^ c[i]) * 1099511628211ull;
  };
  for (auto* g : graphs) mix(&g, sizeof(g));
  for (auto& t : tasks) {
    const size_t n = t.size();
    mix(&n, sizeof(n));
    if (n) mix(t.data(), n * sizeof(bbtc_task));
  }
  mix(&o, sizeof(o));
  std::ostringstream s;
  s << std::hex << h << ":" << graphs.size();
  return s.str();
}

std::vector<bbtc_task> default_tasks(const bbtc_graph* g, bool sorted) {
  uint32_t nt = 0;
  bbtc_task_list(g->P, nullptr, 0, &nt);
  std::vector<bbtc_task> t(nt);
  bbtc_task_list(g->P, t.data(), nt, &nt);
  if (sorted) bbtc_sort_tasks(g, t.data(), nt, 1);
  return t;
}

int finish_upload(bbtc_ctx* ctx, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m,
                  const uint32_t* cuts, uint32_t P, bool host, bbtc_graph** out) {
  bbtc_graph* g = new (std::nothrow) bbtc_graph();
  if (!g) return fail(BBTC_ERR_NOMEM, "host allocation failed");
  g->ctx = ctx;
  g->n = n;
  g->m = m;
  g->P = P;
  g->cuts.assign(cuts, cuts + P + 1);
  if (dev_malloc(&g->d_count, 64 * sizeof(uint64_t), ctx->stream) != cudaSuccess) {
    cudaGetLastError();
    delete g;
    return fail(BBTC_ERR_NOMEM, "device allocation of the result slot failed");
  }
  int rc = build_layout(g, indptr, indices, host);
  if (rc != BBTC_OK) {
    bbtc_graph_free(g);
    return rc;
  }
  *out = g;
  return BBTC_OK;
}

}  // namespace

// Free a graph's device memory on stream s (the caller has made sure nothing
// on the device still reads it) without waiting for the graph's own stream.
void graph_release_on(bbtc_graph* g, cudaStream_t s) {
  if (!g) return;
  for (auto& kv : g->plans) kv.second->release();
  g->fwd.release(s);
  g->rev.release(s);
  if (g->d_indptr) cudaFreeAsync(g->d_indptr, s);
  if (g->d_indices) cudaFreeAsync(g->d_indices, s);
  if (g->d_words) cudaFreeAsync(g->d_words, s);
  if (g->d_wptr) cudaFreeAsync(g->d_wptr, s);
  if (g->d_desc) cudaFreeAsync(g->d_desc, s);
  if (g->d_count) cudaFreeAsync(g->d_count, s);
  delete g;
}

}  // namespace bbtc

using namespace bbtc;

extern "C" {

int bbtc_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return BBTC_ERR_ARG;
  std::snprintf(buf, len, "%s", g_last_error.c_str());
  return BBTC_OK;
}

int bbtc_version(void) { return 10000; }

int bbtc_debug_fail_alloc(int64_t after, int64_t* left) {
  const int64_t prev = g_alloc_fault.exchange(after < 0 ? -1 : after);
  if (left) *left = prev < 0 ? -1 : prev;
  return BBTC_OK;
}

int bbtc_debug_stage_timeout(bbtc_ctx* ctx, uint32_t polls) {
  if (!ctx) return bbtc::fail(BBTC_ERR_ARG, "NULL context");
  ctx->debug_stage_polls = polls;
  return BBTC_OK;
}

int bbtc_ctx_create(int device, bbtc_ctx** out) {
  if (!out) return fail(BBTC_ERR_ARG, "out is NULL");
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(BBTC_ERR_NODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (device < 0 || device >= count) return fail(BBTC_ERR_NODEV, "device index out of range");
  BBTC_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  BBTC_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(BBTC_ERR_NODEV, std::string("device ") + prop.name + " is not sm_100-class; this build targets sm_100a");
  bbtc_ctx* c = new (std::nothrow) bbtc_ctx();
  if (!c) return fail(BBTC_ERR_NOMEM, "host allocation failed");
  c->device = device;
  c->sms = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete c;
    return cuda_fail(e, "cudaStreamCreateWithFlags");
  }
  {
    // keep freed blocks in the device's default pool: repeated uploads reuse them
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  e = dev_malloc_sync(&c->d_unit_counter, 64 * sizeof(uint32_t));
  if (e != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return cuda_fail(e, "cudaMalloc");
  }
  e = cudaMallocHost(&c->h_stage, kStageBytes);
  if (e != cudaSuccess) {
    cudaFree(c->d_unit_counter);
    cudaStreamDestroy(c->stream);
    delete c;
    return cuda_fail(e, "cudaMallocHost");
  }
  *out = c;
  return BBTC_OK;
}

int bbtc_ctx_destroy(bbtc_ctx* ctx) {
  if (!ctx) return BBTC_OK;
  cudaSetDevice(ctx->device);
  if (ctx->d_scratch) cudaFreeAsync(ctx->d_scratch, ctx->stream);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->d_unit_counter) cudaFree(ctx->d_unit_counter);
  if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
  if (ctx->h_plan_done) cudaEventDestroy(ctx->h_plan_done);
  if (ctx->h_plan) cudaFreeHost(ctx->h_plan);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return BBTC_OK;
}

int bbtc_ctx_stream(bbtc_ctx* ctx, void** stream) {
  if (!ctx || !stream) return fail(BBTC_ERR_ARG, "NULL argument");
  *stream = ctx->stream;
  return BBTC_OK;
}

int bbtc_ctx_sm_count(bbtc_ctx* ctx, int* sms) {
  if (!ctx || !sms) return fail(BBTC_ERR_ARG, "NULL argument");
  *sms = ctx->sms;
  return BBTC_OK;
}

int bbtc_ctx_set_zero_copy(bbtc_ctx* ctx, uint64_t max_bytes) {
  if (!ctx) return fail(BBTC_ERR_ARG, "NULL context");
  ctx->zero_copy_bytes = max_bytes;
  return BBTC_OK;
}

int bbtc_graph_upload(bbtc_ctx* ctx, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m,
                      const uint32_t* cuts, uint32_t P, bbtc_graph** out) {
  if (!ctx || !out || !indptr || (m && !indices)) return fail(BBTC_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (m >= (1ull << 32)) return fail(BBTC_ERR_UNSUPPORTED, "m must be below 2^32 (32-bit row pointers)");
  if (n == 0xffffffffu) return fail(BBTC_ERR_ARG, "n must be below 2^32 - 1");
  BBTC_TRY(validate_cuts(n, cuts, P));
  if (indptr[0] != 0 || indptr[n] != m) return fail(BBTC_ERR_INPUT, "indptr[0] must be 0 and indptr[n] must be m");
  BBTC_CUDA(cudaSetDevice(ctx->device));
  return finish_upload(ctx, n, indptr, indices, m, cuts, P, /*host=*/true, out);
}

int bbtc_graph_upload_device(bbtc_ctx* ctx, uint32_t n, const uint32_t* d_indptr, const uint32_t* d_indices,
                             uint64_t m, const uint32_t* cuts, uint32_t P, bbtc_graph** out) {
  if (!ctx || !out || !d_indptr || (m && !d_indices)) return fail(BBTC_ERR_ARG, "NULL argument");
  *out = nullptr;
  if (m >= (1ull << 32)) return fail(BBTC_ERR_UNSUPPORTED, "m must be below 2^32 (32-bit row pointers)");
  if (n == 0xffffffffu) return fail(BBTC_ERR_ARG, "n must be below 2^32 - 1");
  BBTC_TRY(validate_cuts(n, cuts, P));
  BBTC_CUDA(cudaSetDevice(ctx->device));
  return finish_upload(ctx, n, d_indptr, d_indices, m, cuts, P, /*host=*/false, out);
}

int bbtc_graph_free(bbtc_graph* g) {
  if (!g) return BBTC_OK;
  cudaSetDevice(g->ctx->device);
  cudaStreamSynchronize(g->ctx->stream);
  for (auto& kv : g->plans) kv.second->release();
  cudaStream_t s = g->ctx->stream;
  g->fwd.release(s);
  g->rev.release(s);
  if (g->d_indptr) cudaFreeAsync(g->d_indptr, s);
  if (g->d_indices) cudaFreeAsync(g->d_indices, s);
  if (g->d_words) cudaFreeAsync(g->d_words, s);
  if (g->d_wptr) cudaFreeAsync(g->d_wptr, s);
  if (g->d_desc) cudaFreeAsync(g->d_desc, s);
  if (g->d_count) cudaFreeAsync(g->d_count, s);
  cudaStreamSynchronize(s);
  delete g;
  return BBTC_OK;
}

int bbtc_graph_info_get(const bbtc_graph* g, bbtc_graph_info* info) {
  if (!g || !info) return fail(BBTC_ERR_ARG, "NULL argument");
  info->n = g->n;
  info->P = g->P;
  info->m = g->m;
  info->device_bytes = g->device_bytes;
  info->layout_ms = g->layout_ms;
  info->zero_copy = g->zero_copy ? 1u : 0u;
  info->reserved = 0;
  return BBTC_OK;
}

int bbtc_graph_tile_stats(const bbtc_graph* g, uint32_t* nnz, uint32_t* height, uint32_t* width, float* tile_deg,
                          uint32_t* max_deg) {
  if (!g) return fail(BBTC_ERR_ARG, "NULL graph");
  BBTC_TRY(ensure_fwd(const_cast<bbtc_graph*>(g)));
  const uint32_t P = g->P;
  for (uint32_t x = 0; x < P; x++)
    for (uint32_t y = 0; y < P; y++) {
      const uint32_t t = x * P + y;
      const uint32_t H = g->cuts[x + 1] - g->cuts[x];
      if (nnz) nnz[t] = g->fwd.nnz[t];
      if (height) height[t] = H;
      if (width) width[t] = g->cuts[y + 1] - g->cuts[y];
      if (tile_deg) tile_deg[t] = (float)g->fwd.nnz[t] / (float)H;
      if (max_deg) max_deg[t] = g->fwd.maxdeg[t];
    }
  return BBTC_OK;
}

int bbtc_task_list(uint32_t P, bbtc_task* out, uint32_t cap, uint32_t* ntasks) {
  if (!ntasks) return fail(BBTC_ERR_ARG, "ntasks is NULL");
  if (P < 1 || P > kMaxParts) return fail(BBTC_ERR_ARG, "P must be in [1, 64]");
  const uint32_t nt = P * (P + 1) * (P + 2) / 6;
  *ntasks = nt;
  if (!out) return BBTC_OK;
  if (cap < nt) return fail(BBTC_ERR_ARG, "cap is smaller than the task count");
  uint32_t q = 0;
  for (uint32_t i = 0; i < P; i++)
    for (uint32_t j = i; j < P; j++)
      for (uint32_t k = j; k < P; k++) out[q++] = bbtc_task{i * P + j, j * P + k, i * P + k};
  return BBTC_OK;
}

int bbtc_sort_tasks(const bbtc_graph* g, bbtc_task* tasks, uint32_t ntasks, int descending) {
  if (!g || (ntasks && !tasks)) return fail(BBTC_ERR_ARG, "NULL argument");
  const uint32_t P = g->P;
  std::vector<float> deg(P * P);
  BBTC_TRY(bbtc_graph_tile_stats(g, nullptr, nullptr, nullptr, deg.data(), nullptr));
  for (uint32_t q = 0; q < ntasks; q++)
    if (tasks[q].ab >= P * P || tasks[q].bc >= P * P || tasks[q].ac >= P * P)
      return fail(BBTC_ERR_ARG, "task names a tile outside the P x P grid");
  auto weight = [&](const bbtc_task& t) {
    return (float)g->fwd.nnz[t.ab] * std::max(deg[t.bc], deg[t.ac]);
  };
  std::vector<float> w(ntasks);
  for (uint32_t q = 0; q < ntasks; q++) w[q] = weight(tasks[q]);
  std::vector<uint32_t> idx(ntasks);
  std::iota(idx.begin(), idx.end(), 0);
  // NaN weights (empty parts) sort last in either direction
  auto key = [&](uint32_t a) { return std::isnan(w[a]) ? (descending ? -1.0f : 3.4e38f) : w[a]; };
  std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    return descending ? key(a) > key(b) : key(a) < key(b);
  });
  std::vector<bbtc_task> tmp(tasks, tasks + ntasks);
  for (uint32_t q = 0; q < ntasks; q++) tasks[q] = tmp[idx[q]];
  return BBTC_OK;
}

void bbtc_opts_default(bbtc_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->mode = BBTC_MODE_PERSISTENT;
  o->kernel = BBTC_KERNEL_AUTO;
  o->bitmap_words = 0;  // by graph size (count.cu: resolve_opts)
  o->warps_per_block = 8;
  o->unit_work = 0;
  o->blocks_per_sm = 0;
  o->use_cuda_graph = 1;
  o->sort_tasks = 1;
  o->occupancy = 0;  // by bitmap size
}

// Is `tasks` the whole task list of P parts, in any order: every (i <= j <= k)
// exactly once, as (ab, bc, ac) = ((i,j), (j,k), (i,k))?
static bool is_full_task_list(uint32_t P, const bbtc_task* tasks, uint32_t ntasks) {
  if (ntasks != P * (P + 1) * (P + 2) / 6) return false;
  std::vector<uint8_t> seen((size_t)P * P * P, 0);
  for (uint32_t q = 0; q < ntasks; q++) {
    const bbtc_task& t = tasks[q];
    if (t.ab >= P * P || t.bc >= P * P) return false;
    const uint32_t i = t.ab / P, j = t.ab % P, k = t.bc % P;
    if (t.bc / P != j || t.ac != i * P + k || i > j || j > k) return false;
    uint8_t& s = seen[((size_t)i * P + j) * P + k];
    if (s) return false;
    s = 1;
  }
  return true;
}

static int count_async_impl(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_task* tasks, uint32_t ntasks, int32_t border,
                            const bbtc_opts* opts) {
  if (!ctx || !g) return fail(BBTC_ERR_ARG, "NULL argument");
  if (g->ctx != ctx) return fail(BBTC_ERR_ARG, "graph belongs to another context");
  if (border < -1) return fail(BBTC_ERR_ARG, "border must be -1 or >= 0");
  bbtc_opts o;
  if (opts) o = *opts; else bbtc_opts_default(&o);
  if (o.mode != BBTC_MODE_PLAIN && o.mode != BBTC_MODE_PERSISTENT) return fail(BBTC_ERR_ARG, "unknown mode");
  if (o.kernel < BBTC_KERNEL_AUTO || o.kernel > BBTC_KERNEL_FUSED) return fail(BBTC_ERR_ARG, "unknown kernel");
  // The fused task rows count the whole task list at once.  A caller that
  // passes the whole list (the reference's driver does, in its cost order)
  // gets them too: the sum does not depend on the order, and with one device
  // queue the border only orders the queue.
  const bool whole = !tasks || is_full_task_list(g->P, tasks, ntasks);
  if (o.kernel == BBTC_KERNEL_FUSED && !whole)
    return fail(BBTC_ERR_ARG, "fused task rows run the whole task list: pass tasks = NULL or every task once");
  const bool fused = whole && (o.kernel == BBTC_KERNEL_FUSED ||
                               (o.kernel == BBTC_KERNEL_AUTO && o.mode == BBTC_MODE_PERSISTENT));
  BBTC_CUDA(cudaSetDevice(ctx->device));
  if (!fused) BBTC_TRY(ensure_fwd(g));  // task-list counting reads the forward block CSR
  std::vector<std::vector<bbtc_task>> tl(1);
  // fused task rows run every task whatever the order: no sort (it would need the forward tiles)
  if (tasks) tl[0].assign(tasks, tasks + ntasks); else tl[0] = default_tasks(g, !fused && o.sort_tasks != 0);
  // border b >= 0: tasks [0, b) are queued ahead of the rest; with one device queue in list
  // order that is the list order itself, so the value only has to be in range.
  std::vector<bbtc_graph*> gs{g};
  const std::string key = plan_key(gs, tl, o);
  auto it = g->plans.find(key);
  const bool reuse = it != g->plans.end();
  if (!reuse) {
    if (g->plans.size() > 16) {
      for (auto& kv : g->plans) kv.second->release();
      g->plans.clear();
    }
    it = g->plans.emplace(key, std::make_unique<Plan>()).first;
  }
  const int rc = count_enqueue(ctx, gs, tl, o, fused, g->d_count, it->second.get(), reuse);
  if (rc != BBTC_OK) {
    it->second->release();
    g->plans.erase(it);
    return rc;
  }
  g->last_launches = it->second->launches;
  return BBTC_OK;
}

int bbtc_count_async(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_task* tasks, uint32_t ntasks, int32_t border,
                     const bbtc_opts* opts) {
  return count_async_impl(ctx, g, tasks, ntasks, border, opts);
}

int bbtc_count_wait(bbtc_ctx* ctx, bbtc_graph* g, uint64_t* out) {
  Range range("bbtc count wait");
  if (!ctx || !g || !out) return fail(BBTC_ERR_ARG, "NULL argument");
  BBTC_CUDA(cudaSetDevice(ctx->device));
  uint64_t* h = reinterpret_cast<uint64_t*>(ctx->h_stage + kStageOut);
  BBTC_CUDA(cudaMemcpyAsync(h, g->d_count, sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BBTC_TRY(staging_status(ctx));  // synchronises the stream
  *out = *h;
  return BBTC_OK;
}

int bbtc_count(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_task* tasks, uint32_t ntasks, int32_t border,
               const bbtc_opts* opts, uint64_t* out) {
  if (!out) return fail(BBTC_ERR_ARG, "out is NULL");
  BBTC_TRY(count_async_impl(ctx, g, tasks, ntasks, border, opts));
  return bbtc_count_wait(ctx, g, out);
}

int bbtc_last_launches(const bbtc_graph* g, uint32_t* launches) {
  if (!g || !launches) return fail(BBTC_ERR_ARG, "NULL argument");
  *launches = g->last_launches;
  return BBTC_OK;
}

int bbtc_autotune(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_tune_space* space, bbtc_opts* inout, double* best_ms) {
  if (!ctx || !g || !inout) return fail(BBTC_ERR_ARG, "NULL argument");
  static const uint32_t kWords[] = {256, 512, 1024, 2048, 4096};
  static const uint32_t kWarps[] = {4, 8};
  static const uint32_t kWork[] = {256, 2048, 8192};
  static const uint32_t kOcc[] = {4, 6, 8};
  bbtc_tune_space sp{kWords, 5, kWarps, 2, kWork, 3, 3, kOcc, 3};
  if (space) {
    sp = *space;
    if (!sp.occupancy || !sp.n_occupancy) { sp.occupancy = kOcc; sp.n_occupancy = 3; }
    if (!sp.bitmap_words || !sp.n_bitmap_words) { sp.bitmap_words = kWords; sp.n_bitmap_words = 5; }
    if (!sp.warps_per_block || !sp.n_warps_per_block) { sp.warps_per_block = kWarps; sp.n_warps_per_block = 2; }
    if (!sp.unit_work || !sp.n_unit_work) { sp.unit_work = kWork; sp.n_unit_work = 3; }
    if (!sp.repeats) sp.repeats = 3;
  }
  BBTC_CUDA(cudaSetDevice(ctx->device));
  cudaEvent_t a, b;
  BBTC_CUDA(cudaEventCreate(&a));
  BBTC_CUDA(cudaEventCreate(&b));
  struct Ev {
    cudaEvent_t a, b;
    ~Ev() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } evs{a, b};
  bbtc_opts best = *inout;
  double best_t = 1e300;
  uint64_t ref_count = 0;
  bool have_ref = false;
  for (uint32_t iw = 0; iw < sp.n_bitmap_words; iw++)
    for (uint32_t ip = 0; ip < sp.n_warps_per_block; ip++)
      for (uint32_t iu = 0; iu < sp.n_unit_work; iu++)
      for (uint32_t io = 0; io < sp.n_occupancy; io++) {
        bbtc_opts o = *inout;
        o.bitmap_words = sp.bitmap_words[iw];
        o.warps_per_block = sp.warps_per_block[ip];
        o.unit_work = sp.unit_work[iu];
        o.occupancy = sp.occupancy[io];
        if (smem_bytes_for(o) > ctx->smem_optin) continue;  // does not fit this device
        uint64_t c = 0;
        BBTC_TRY(bbtc_count(ctx, g, nullptr, 0, -1, &o, &c));  // warm-up, builds the plan
        std::vector<float> ts;
        for (uint32_t r = 0; r < sp.repeats; r++) {
          BBTC_CUDA(cudaEventRecord(a, ctx->stream));
          BBTC_TRY(bbtc_count_async(ctx, g, nullptr, 0, -1, &o));
          BBTC_CUDA(cudaEventRecord(b, ctx->stream));
          BBTC_TRY(bbtc_count_wait(ctx, g, &c));
          float ms = 0;
          BBTC_CUDA(cudaEventElapsedTime(&ms, a, b));
          ts.push_back(ms);
          if (!have_ref) {
            ref_count = c;
            have_ref = true;
          } else if (c != ref_count) {
            return fail(BBTC_ERR_STATE, "autotune points disagree on the count");
          }
        }
        std::sort(ts.begin(), ts.end());
        const double med = ts[ts.size() / 2];
        if (med < best_t) {
          best_t = med;
          best = o;
        }
      }
  if (!have_ref) return fail(BBTC_ERR_ARG, "no point of the tuning space fits this device");
  *inout = best;
  if (best_ms) *best_ms = best_t;
  return BBTC_OK;
}

int bbtc_count_batch(bbtc_ctx* ctx, bbtc_graph* const* graphs, uint32_t ng, const bbtc_opts* opts, uint64_t* outs) {
  Range range("bbtc count batch");
  if (!ctx || (ng && (!graphs || !outs))) return fail(BBTC_ERR_ARG, "NULL argument");
  if (ng == 0) return BBTC_OK;
  bbtc_opts o;
  if (opts) o = *opts; else bbtc_opts_default(&o);
  if (o.mode != BBTC_MODE_PERSISTENT && o.mode != BBTC_MODE_PLAIN) return fail(BBTC_ERR_ARG, "unknown mode");
  if (o.kernel < BBTC_KERNEL_AUTO || o.kernel > BBTC_KERNEL_FUSED) return fail(BBTC_ERR_ARG, "unknown kernel");
  BBTC_CUDA(cudaSetDevice(ctx->device));
  std::vector<bbtc_graph*> gs(graphs, graphs + ng);
  std::vector<std::vector<bbtc_task>> tl(ng);
  const bool fused_all = o.kernel == BBTC_KERNEL_FUSED || (o.kernel == BBTC_KERNEL_AUTO && o.mode == BBTC_MODE_PERSISTENT);
  for (uint32_t i = 0; i < ng; i++) {
    if (!gs[i] || gs[i]->ctx != ctx) return fail(BBTC_ERR_ARG, "graph is NULL or belongs to another context");
    if (!fused_all) BBTC_TRY(ensure_fwd(gs[i]));
    tl[i] = default_tasks(gs[i], !fused_all && o.sort_tasks != 0);
  }
  uint64_t* d_outs = nullptr;
  BBTC_CUDA(dev_malloc(&d_outs, ng * sizeof(uint64_t), ctx->stream));
  struct F {
    uint64_t* p;
    cudaStream_t s;
    ~F() { cudaFreeAsync(p, s); }
  } guard{d_outs, ctx->stream};
  Plan plan;
  o.use_cuda_graph = 0;
  // one queue for all graphs: tasks of every graph merged by cost, heaviest first
  const bool fused = o.kernel == BBTC_KERNEL_FUSED || (o.kernel == BBTC_KERNEL_AUTO && o.mode == BBTC_MODE_PERSISTENT);
  int rc = count_enqueue(ctx, gs, tl, o, fused, d_outs, &plan, false);
  if (rc == BBTC_OK) {
    const bool staged = (size_t)ng * sizeof(uint64_t) <= kStageBytes - kStageOut;
    uint64_t* h = staged ? reinterpret_cast<uint64_t*>(ctx->h_stage + kStageOut) : outs;
    cudaError_t e = cudaMemcpyAsync(h, d_outs, ng * sizeof(uint64_t), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) rc = cuda_fail(e, "batch readback");
    else rc = staging_status(ctx);
    if (rc == BBTC_OK && staged) std::memcpy(outs, h, ng * sizeof(uint64_t));
  }
  for (uint32_t i = 0; i < ng; i++) gs[i]->last_launches = plan.launches;
  plan.release();
  return rc;
}

}  // extern "C"

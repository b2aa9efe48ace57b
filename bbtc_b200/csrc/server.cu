// Request server: continuous batching of count requests on one GPU.
//
// No counterpart in the reference (it counts one graph per process).  A
// request is a host CSR + cut vector; its answer is the exact count.
//
//   loader threads (each with its own stream): take the oldest pending
//     request whose estimated device footprint fits the HBM budget, build its
//     device block CSR (upload + layout), mark it ready.  A request that could
//     never fit fails with BBTC_ERR_CAPACITY.
//   launcher thread (its own stream): takes every ready graph (up to
//     max_batch), counts them in one persistent launch with one u64 slot per
//     graph, publishes the counts, frees the graphs, returns their memory to
//     the budget.
//
// So requests that arrive while a launch is on the GPU are uploaded and laid
// out on the loader streams at the same time, and join the next launch; the
// device always holds the graphs being counted plus those being loaded.
// Every result is written to its own slot, so a graph's count does not depend
// on what shares its launch.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

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

struct bbtc_server {
  bbtc_server_opts opts{};
  int device = 0;
  std::vector<bbtc_ctx*> load_ctx;
  bbtc_ctx* run_ctx = nullptr;
  std::mutex mu;
  std::condition_variable cv_load, cv_run, cv_done;
  std::deque<bbtc::Request*> pending;
  std::deque<bbtc::Request*> ready;
  std::unordered_map<uint64_t, bbtc::Request*> all;
  uint64_t next_id = 1;
  uint64_t in_use = 0;
  uint32_t loading = 0;
  bool stop = false;
  std::vector<std::thread> loaders;
  std::thread launcher;
  uint64_t* d_outs = nullptr;
  std::vector<uint64_t> h_outs;
  // statistics
  uint64_t launches = 0, counted = 0, max_batch_seen = 0;
};

namespace bbtc {
namespace {

void loader_main(bbtc_server* s, bbtc_ctx* ctx) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    s->cv_load.wait(lk, [&] {
      if (s->stop) return true;
      if (s->pending.empty()) return false;
      const Request* r = s->pending.front();
      return s->in_use + r->reserved <= s->opts.hbm_budget || (s->in_use == 0);
    });
    if (s->stop) return;
    Request* r = s->pending.front();
    s->pending.pop_front();
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
    lk.unlock();
    bbtc_graph* g = nullptr;
    const int rc = bbtc_graph_upload(ctx, r->n, r->indptr, r->indices, r->m, r->cuts.data(),
                                     (uint32_t)r->cuts.size() - 1, &g);
    lk.lock();
    s->loading--;
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
    s->ready.push_back(r);
    s->cv_run.notify_one();
    s->cv_load.notify_all();
  }
}

void launcher_main(bbtc_server* s) {
  cudaSetDevice(s->device);
  bbtc_ctx* ctx = s->run_ctx;
  std::unique_lock<std::mutex> lk(s->mu);
  Plan plan;
  while (true) {
    s->cv_run.wait(lk, [&] { return s->stop || !s->ready.empty(); });
    if (s->stop && s->ready.empty()) break;
    std::vector<Request*> batch;
    while (!s->ready.empty() && batch.size() < s->opts.max_batch) {
      batch.push_back(s->ready.front());
      s->ready.pop_front();
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
    const bool fused = o.kernel == BBTC_KERNEL_FUSED || (o.kernel == BBTC_KERNEL_AUTO && o.mode == BBTC_MODE_PERSISTENT);
    int rc = BBTC_OK;
    if (!fused) {
      for (size_t i = 0; i < batch.size(); i++) {
        uint32_t nt = 0;
        bbtc_task_list(gs[i]->P, nullptr, 0, &nt);
        tl[i].resize(nt);
        bbtc_task_list(gs[i]->P, tl[i].data(), nt, &nt);
      }
    }
    rc = count_enqueue(ctx, gs, tl, o, fused, s->d_outs, &plan, false);
    if (rc == BBTC_OK) {
      const cudaError_t e =
          cudaMemcpyAsync(s->h_outs.data(), s->d_outs, batch.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                          ctx->stream);
      const cudaError_t e2 = e == cudaSuccess ? cudaStreamSynchronize(ctx->stream) : e;
      if (e2 != cudaSuccess) rc = cuda_fail(e2, "server batch readback");
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
        r->count = s->h_outs[i];
        r->status = 4;
      } else {
        r->status = rc;
      }
    }
    s->launches++;
    s->counted += batch.size();
    s->max_batch_seen = std::max<uint64_t>(s->max_batch_seen, batch.size());
    s->cv_done.notify_all();
    s->cv_load.notify_all();
  }
  lk.unlock();
  plan.release();
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
  o->loaders = 2;
  bbtc_opts_default(&o->count);
}

int bbtc_server_create(int device, const bbtc_server_opts* opts, bbtc_server** out) {
  if (!out) return fail(BBTC_ERR_ARG, "out is NULL");
  *out = nullptr;
  bbtc_server* s = new (std::nothrow) bbtc_server();
  if (!s) return fail(BBTC_ERR_NOMEM, "host allocation failed");
  if (opts) s->opts = *opts; else bbtc_server_opts_default(&s->opts);
  if (!s->opts.hbm_budget) s->opts.hbm_budget = 150ull << 30;
  if (!s->opts.max_batch) s->opts.max_batch = 4096;
  if (!s->opts.max_requests) s->opts.max_requests = 1u << 20;
  if (!s->opts.loaders) s->opts.loaders = 2;
  s->opts.loaders = std::min<uint32_t>(s->opts.loaders, 16);
  s->device = device;
  int rc = bbtc_ctx_create(device, &s->run_ctx);
  for (uint32_t i = 0; rc == BBTC_OK && i < s->opts.loaders; i++) {
    bbtc_ctx* c = nullptr;
    rc = bbtc_ctx_create(device, &c);
    if (rc == BBTC_OK) s->load_ctx.push_back(c);
  }
  if (rc == BBTC_OK && cudaMalloc(&s->d_outs, s->opts.max_batch * sizeof(uint64_t)) != cudaSuccess) {
    cudaGetLastError();
    rc = fail(BBTC_ERR_NOMEM, "device allocation of the result slots failed");
  }
  if (rc != BBTC_OK) {
    for (auto* c : s->load_ctx) bbtc_ctx_destroy(c);
    if (s->run_ctx) bbtc_ctx_destroy(s->run_ctx);
    if (s->d_outs) cudaFree(s->d_outs);
    delete s;
    return rc;
  }
  s->h_outs.assign(s->opts.max_batch, 0);
  for (auto* c : s->load_ctx) s->loaders.emplace_back(loader_main, s, c);
  s->launcher = std::thread(launcher_main, s);
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
    s->cv_run.notify_all();
  }
  for (auto& t : s->loaders) t.join();
  s->launcher.join();
  for (auto& kv : s->all) {
    if (kv.second->g) graph_release_on(kv.second->g, s->run_ctx->stream);
    delete kv.second;
  }
  cudaSetDevice(s->device);
  cudaFree(s->d_outs);
  for (auto* c : s->load_ctx) bbtc_ctx_destroy(c);
  bbtc_ctx_destroy(s->run_ctx);
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
  s->cv_load.notify_one();
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
  st->launches = s->launches;
  st->counted = s->counted;
  st->max_batch = s->max_batch_seen;
  st->pending = s->pending.size();
  st->ready = s->ready.size();
  st->device_bytes_in_use = s->in_use;
  return BBTC_OK;
}

}  // extern "C"

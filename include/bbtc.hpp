// bbtc.hpp -- C++ mirror of the reference's host classes over the C ABI.
//
// Same class and method names as GT-TDAlab/bbTC's driver objects so a caller
// of the reference switches by changing includes:
//   BlockCSR  include/data_structures/block_csr.h:19-231  -> device-resident layout
//   tasks::TaskList / SortTasks  include/utils/tasks.hpp:7-34
//   BBTc      include/triangle_counting/bb_tc.h:28-218   -> GPU-only driver
// Errors: the C ABI never exits; these wrappers throw bbtc::Error carrying the
// status and message (the reference has no error reporting at all).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "bbtc_gpu.h"

namespace bbtc {

class Error : public std::runtime_error {
 public:
  Error(int status, const std::string& msg) : std::runtime_error(msg), status_(status) {}
  int status() const { return status_; }

 private:
  int status_;
};

inline void check(int rc) {
  if (rc != BBTC_OK) {
    char buf[1024];
    bbtc_last_error(buf, sizeof(buf));
    throw Error(rc, buf);
  }
}

// One device + stream.
class Context {
 public:
  explicit Context(int device = 0) { check(bbtc_ctx_create(device, &h_)); }
  ~Context() { bbtc_ctx_destroy(h_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  bbtc_ctx* get() const { return h_; }

 private:
  bbtc_ctx* h_ = nullptr;
};

// The block CSR, built on and kept in device memory.
class BlockCSR {
 public:
  BlockCSR(Context& ctx, const std::vector<uint32_t>& cuts, const std::vector<uint32_t>& x_adj,
           const std::vector<uint32_t>& adj)
      : n_((uint32_t)x_adj.size() - 1), m_(adj.size()), cuts_(cuts) {
    check(bbtc_graph_upload(ctx.get(), n_, x_adj.data(), adj.empty() ? nullptr : adj.data(), m_, cuts.data(),
                            (uint32_t)cuts.size() - 1, &g_));
  }
  ~BlockCSR() { CleanUp(); }
  BlockCSR(const BlockCSR&) = delete;
  BlockCSR& operator=(const BlockCSR&) = delete;

  void CleanUp() {
    if (g_) bbtc_graph_free(g_);
    g_ = nullptr;
  }
  uint32_t GetNoOfCuts() const { return (uint32_t)cuts_.size() - 1; }
  uint32_t GetNoOfTiles() const { return GetNoOfCuts() * GetNoOfCuts(); }
  uint32_t GetNoOfVertices() const { return n_; }
  uint64_t GetNoOfEdges() const { return m_; }
  const std::vector<uint32_t>& GetCuts() const { return cuts_; }
  double LayoutMs() const {
    bbtc_graph_info i;
    check(bbtc_graph_info_get(g_, &i));
    return i.layout_ms;
  }
  bbtc_graph* get() const { return g_; }

 private:
  uint32_t n_;
  uint64_t m_;
  std::vector<uint32_t> cuts_;
  bbtc_graph* g_ = nullptr;
};

namespace tasks {
inline std::vector<bbtc_task> TaskList(uint32_t P) {
  uint32_t nt = 0;
  check(bbtc_task_list(P, nullptr, 0, &nt));
  std::vector<bbtc_task> t(nt);
  check(bbtc_task_list(P, t.data(), nt, &nt));
  return t;
}
// Descending cost order, as the reference's CUDA build sorts (tasks.hpp:25-28).
inline void SortTasks(std::vector<bbtc_task>& t, const BlockCSR& st) {
  check(bbtc_sort_tasks(st.get(), t.data(), (uint32_t)t.size(), 1));
}
}  // namespace tasks

// The counting driver.  Separator keeps --border's meaning (tasks [0, b)
// first).  Every task runs on the GPU unless SetCpuWorkers adds CPU workers:
// then tasks [0, Separator) stay on the GPU and the rest are shared, CPU
// workers taking them from the tail (bb_tc.cpp:142-252).
class BBTc {
 public:
  BBTc(Context& ctx, BlockCSR* st, std::vector<bbtc_task>& tasks, uint32_t P)
      : ctx_(ctx), st_(st), tasks_(tasks) {
    if (P != st->GetNoOfCuts()) throw Error(BBTC_ERR_ARG, "P does not match the block CSR");
    bbtc_opts_default(&opts_);
  }
  int Separator = -1;

  void InitFlags() {}
  void ResetFlags() {}
  void PrepareGpu() {}
  void CopyTilesToGpu() {}  // tiles are resident from upload on
  void SetNGPU(int n) {
    if (n != 1) throw Error(BBTC_ERR_UNSUPPORTED, "one GPU is served (--ngpu 1)");
  }
  int GetNGPU() const { return 1; }
  bbtc_opts& Options() { return opts_; }
  // k CPU workers beside the GPU (0 = GPU only).  They read the host CSR the
  // BlockCSR was built from; x_adj and adj must stay alive and unchanged
  // while NoOfTriangles runs.
  void SetCpuWorkers(uint32_t k, const std::vector<uint32_t>& x_adj, const std::vector<uint32_t>& adj) {
    cpu_workers_ = k;
    x_adj_ = x_adj.data();
    adj_ = adj.data();
  }
  const bbtc_hybrid_stats& LastHybridStats() const { return stats_; }

  unsigned long long NoOfTriangles() {
    uint64_t out = 0;
    if (cpu_workers_ > 0) {
      const int32_t border = Separator < -2 ? -1 : Separator;
      check(bbtc_count_hybrid(ctx_.get(), st_->get(), x_adj_, adj_, tasks_.data(), (uint32_t)tasks_.size(), border,
                              cpu_workers_, &opts_, &out, &stats_));
      return out;
    }
    const int32_t border = (Separator < 0 || Separator >= (int)tasks_.size()) ? -1 : Separator;
    check(bbtc_count(ctx_.get(), st_->get(), tasks_.data(), (uint32_t)tasks_.size(), border, &opts_, &out));
    return out;
  }
  void CleanUp() {}

 private:
  Context& ctx_;
  BlockCSR* st_;
  std::vector<bbtc_task> tasks_;
  bbtc_opts opts_;
  uint32_t cpu_workers_ = 0;
  const uint32_t* x_adj_ = nullptr;
  const uint32_t* adj_ = nullptr;
  bbtc_hybrid_stats stats_{};
};

}  // namespace bbtc

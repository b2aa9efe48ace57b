// Internal structures shared by the translation units of libbbtc.so.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/bbtc_gpu.h"

namespace bbtc {

// ---- errors ---------------------------------------------------------------
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define BBTC_CUDA(call)                                   \
  do {                                                    \
    cudaError_t e__ = (call);                             \
    if (e__ != cudaSuccess) return ::bbtc::cuda_fail(e__, #call); \
  } while (0)

#define BBTC_TRY(call)          \
  do {                          \
    int rc__ = (call);          \
    if (rc__ != BBTC_OK) return rc__; \
  } while (0)

// ---- device allocations ---------------------------------------------------
// Every device allocation of the library whose failure is an error goes
// through dev_malloc / dev_malloc_sync, so that a test hook
// (bbtc_debug_fail_alloc, or BBTC_FAIL_ALLOC=k in the environment when the
// library loads) can make the k-th next one fail as if the device were out of
// memory.  take_alloc_fault() consumes the armed fault (true once, when the
// count reaches it).
bool take_alloc_fault();

template <class T>
inline cudaError_t dev_malloc(T** p, size_t bytes, cudaStream_t s) {
  if (take_alloc_fault()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocAsync(reinterpret_cast<void**>(p), bytes, s);
}

template <class T>
inline cudaError_t dev_malloc_sync(T** p, size_t bytes) {
  if (take_alloc_fault()) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

// A named range on the NVTX timeline (shown by nsys, filterable in ncu with
// --nvtx); with no tool attached it costs a pointer check.
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
  Range(const Range&) = delete;
  Range& operator=(const Range&) = delete;
};

constexpr uint32_t kMaxParts = 64;
constexpr uint32_t kMaxDevices = 64;
constexpr uint64_t kNoSegment = ~0ull;

// One tile as the kernels see it: tile-local row pointers (H+1 entries, the
// first is 0) and tile-local column ids, both 16-byte aligned.  An empty tile
// has rp == nullptr.
struct DevTile {
  const uint32_t* rp;
  const uint32_t* col;
  const uint2* rec;  // reversed tiles: pair range [word of v, end) in row u, per entry's forward edge (u, v)
  const uint32_t* erow;  // row of entry 32 q, for q < ceil(nnz / 32)
  uint32_t H, W, nnz, maxdeg;
};

// Kinds of work a task is run as (see count.cu).
enum TaskKind : uint32_t {
  kPivotBitmap = 0,  // pivot row -> shared bitmap of the column part, probes test bits
  kPivotList = 1,    // pivot row -> sorted shared list, probes binary-search it
  kPivotGlobal = 2,  // pivot row too long for shared memory: binary search in global memory
  kFusedRow = 3,     // task row (i, j): all tasks (i, j, k >= j) in one pass, structure chosen per pivot
  kPivotSplit = 4,   // pivot row -> bitmap of its top id window + short sorted list of the ids below it
  kPivotRank = 5,    // fused task rows: per 32-word block of the row's span a (presence bits, first pair)
                     // entry, then the row's masks in pair order (a rank bitmap over the words)
};

// One queued task: `rows` is the tile whose rows are the pivot vertices and
// whose entries select the probe rows; `pivot` holds the pivot vertices' rows
// (the set each intersection is tested against) and `probe` the rows that
// are streamed against it.  For the v-centric order rows = CSC of ab
// (reversed tile (j,i)), pivot = bc, probe = ac.  For the u-centric order
// (the reference's row order) rows = ab, pivot = ac, probe = bc.
struct DevTask {
  DevTile rows;
  DevTile pivot;
  DevTile probe;
  const uint32_t* g_indptr;   // fused task rows: the resident oriented CSR
  const uint32_t* g_indices;
  const uint2* g_words;       // fused: word-compressed rows
  const uint32_t* g_wptr;     // fused: their row pointers (n + 1)
  const uint4* g_desc;        // fused: per vertex (row start, pair start, first id, last id), n + 1
  uint32_t pivot_base;        // fused: first vertex id of part j
  uint32_t kind;
  uint32_t unit_edges;  // entries of `rows` per work unit
  uint32_t slot;        // output counter index
  uint32_t words;       // bitmap words the pivot part needs (ceil(W/32))
};

// A block CSR over one cut vector, for the forward or the reversed graph.
struct BlockTiles {
  uint32_t P = 0;
  std::vector<uint32_t> nnz, maxdeg, nerows;  // P*P each
  std::vector<uint64_t> rp_off, col_off;      // element offsets, kNoSegment when empty
  uint32_t* d_rp = nullptr;                    // row-pointer pool
  uint32_t* d_col = nullptr;                   // column pool
  void* d_rec = nullptr;                       // reversed tiles: forward-edge records (uint2), col-aligned
  uint32_t* d_erow = nullptr;                  // row index of every 32nd entry, per tile
  size_t rp_len = 0, col_len = 0, erow_len = 0;
  cudaStream_t stream = nullptr;
  void release(cudaStream_t s);
};

struct Plan {
  std::vector<DevTask> tasks;      // host copy
  std::vector<uint32_t> prefix;    // unit prefix, ntasks + 1
  DevTask* d_tasks = nullptr;      // stream-ordered, reused while large enough
  uint32_t* d_prefix = nullptr;
  size_t cap = 0;                  // tasks the device buffers hold
  cudaStream_t stream = nullptr;   // stream the buffers were allocated on
  uint32_t total_units = 0;
  uint32_t launches = 0;
  bool fused = false;              // every task is a fused task row
  cudaGraphExec_t exec = nullptr;
  bool captured = false;
  uint32_t stage_polls = 0;        // the context's staging test hook when the launch was captured
  void release();
};

}  // namespace bbtc

struct bbtc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sms = 0;
  size_t smem_optin = 0;
  uint32_t* d_unit_counter = nullptr;  // persistent-queue head (one word per launch slot)
  size_t smem_set = 0;                 // dynamic shared memory the count kernels are opted in to
  bool open_carveout = false;          // layout kernels ask for the largest shared-memory carveout (launch_layout)
  uint32_t layout_blocks_per_sm = 8;   // grid cap of the layout kernels (256 threads a block)
  uint32_t upload_window = 0;          // host uploads: pieces in flight at most (0 = all at once)
  uint64_t zero_copy_bytes = 0;        // host arrays up to this size in mapped page-locked memory are read
                                       // by a kernel instead of the copy engines (0 = never)
  uint32_t debug_stage_polls = 0;      // test hook (bbtc_debug_stage_timeout): > 0 = staging copies are not
                                       // issued and their waits give up after this many polls
  // Page-locked staging for the small control copies (cut vectors, tile
  // offsets and statistics, counts).  A copy to or from pageable memory is
  // staged by the driver through buffers every thread shares, so one that
  // waited for a long kernel on its stream held up the copies of all other
  // threads; copies from pinned memory wait only for their own stream.
  char* h_stage = nullptr;
  // Pinned staging of the task queues' uploads, kept across plans.
  char* h_plan = nullptr;
  size_t h_plan_cap = 0;
  cudaEvent_t h_plan_done = nullptr;  // recorded after the last upload from h_plan
  // Layout scratch kept between builds (bbtc::Scratch), at most kScratchKeep bytes.
  char* d_scratch = nullptr;
  size_t scratch_cap = 0;
};

namespace bbtc {

// Scratch of one layout build: its temporaries are carved from one device
// block that the context keeps between builds, so a build whose temporaries
// fit makes no allocation call for them.  `want` sums what the build asked
// for (256-byte rounded), carved or not; the block grows to it afterwards.
struct Scratch {
  char* base = nullptr;
  size_t cap = 0, off = 0, want = 0;
};
// The build running on this thread, if any (one build at a time per context,
// and a context's builds run on the thread that called them).
inline thread_local Scratch* t_scratch = nullptr;

// Stream-ordered device buffer (freed on the stream it was allocated on);
// carved from the running build's scratch when that has room.
struct DevBuf {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  bool carved = false;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p && !carved) cudaFreeAsync(p, s);
  }
  template <class T>
  T* as() { return static_cast<T*>(p); }
};

inline int dalloc(DevBuf& b, size_t bytes, cudaStream_t s) {
  b.s = s;
  if (Scratch* a = t_scratch) {
    const size_t need = ((bytes > 16 ? bytes : 16) + 255) & ~static_cast<size_t>(255);
    a->want += need;
    if (a->off + need <= a->cap) {
      b.p = a->base + a->off;
      b.carved = true;
      a->off += need;
      return BBTC_OK;
    }
  }
  cudaError_t e = dev_malloc(&b.p, bytes > 16 ? bytes : 16, s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return fail(BBTC_ERR_NOMEM, std::string("device allocation of ") + std::to_string(bytes) +
                                    " bytes failed: " + cudaGetErrorString(e));
  }
  return BBTC_OK;
}

// Regions of bbtc_ctx::h_stage (one graph build or count at a time per context).
constexpr size_t kStageBytes = 1u << 20;
constexpr size_t kStageCuts = 0;          // cut vector and a flags word, <= (64 + 2) x 4 bytes
constexpr size_t kStageBad = 3072;        // validation flags
constexpr size_t kStageOff[2] = {4096, 40960};  // per block CSR: tile + part row offsets (<= 33,288 bytes)
constexpr size_t kStageStats = 81920;     // tile statistics of both block CSRs (<= 163,840 bytes)
constexpr size_t kStageOut = 262144;      // counts read back (<= 98,304 of them)

}  // namespace bbtc

struct bbtc_graph {
  bbtc_ctx* ctx = nullptr;
  uint32_t n = 0, P = 0;
  uint64_t m = 0;
  std::vector<uint32_t> cuts;
  uint32_t* d_indptr = nullptr;   // resident oriented CSR (global ids)
  uint32_t* d_indices = nullptr;
  void* d_words = nullptr;        // word-compressed rows: (word, mask) uint2 pairs
  uint32_t* d_wptr = nullptr;     // n + 1 pair offsets
  void* d_desc = nullptr;         // n + 1 pivot descriptors (uint4): row start, pair start, first id, last id
  bbtc::BlockTiles fwd, rev;
  uint64_t* d_count = nullptr;  // result slot
  uint64_t device_bytes = 0;
  double layout_ms = 0;
  bool fwd_built = false;         // the forward block CSR is built on first use (task-list counting, tile stats)
  bool zero_copy = false;         // the upload read the host CSR with a kernel (no copy-engine transfer)
  uint32_t last_launches = 0;
  std::map<std::string, std::unique_ptr<bbtc::Plan>> plans;  // cached queues keyed by request
};

namespace bbtc {

// layout.cu
// indptr / indices are host memory when `host`, else device memory of the
// context's device; the graph keeps its own device copy either way.
int build_layout(bbtc_graph* g, const uint32_t* indptr, const uint32_t* indices, bool host);
// Build g's forward block CSR if it is not built yet (on g's context stream; synchronises it).
int ensure_fwd(bbtc_graph* g);
DevTile dev_tile(const BlockTiles& t, const std::vector<uint32_t>& cuts, uint32_t x, uint32_t y);

// count.cu
int count_enqueue(bbtc_ctx* ctx, const std::vector<bbtc_graph*>& graphs,
                  const std::vector<std::vector<bbtc_task>>& tasks, const bbtc_opts& o, bool fused,
                  uint64_t* d_outs, Plan* plan, bool reuse);
int kernel_smem_optin(bbtc_ctx* ctx, const bbtc_opts& o);
// After a count has finished on ctx's stream: BBTC_ERR_TIMEOUT if a
// shared-memory staging copy of the launch gave up waiting (the count is void).
int staging_status(bbtc_ctx* ctx);
size_t smem_bytes_for(const bbtc_opts& o);

}  // namespace bbtc

/*
 * bbtc_gpu.h -- C ABI of the B200 triangle-counting path (libbbtc.so).
 *
 * Exact triangle counting over a 2D-partitioned block CSR, task model
 * (i <= j <= k) as in GT-TDAlab/bbTC.  Every function returns an int status:
 * 0 (BBTC_OK) or a negative bbtc_status; bbtc_last_error() gives the message
 * of the calling thread's last failure.  No function exits the process.
 *
 * Reference interfaces each entry point replaces (paths inside the bbTC
 * project):
 *   - class BBTc                         include/triangle_counting/bb_tc.h:28-218
 *   - BlockCSR(cuts, x_adj, adj)         src/data_structures/block_csr.cpp:35-42, 288-376
 *   - tasks::TaskList / tasks::SortTasks include/utils/tasks.hpp:7-34
 *   - DenseKernel / SparseKernel launch  src/triangle_counting/bb_tc.cpp:76-115
 *   - BBTc::NoOfTriangles                src/triangle_counting/bb_tc.cpp:200-252
 *   - RunGpuKernels / RunCpuKernels      src/triangle_counting/bb_tc.cpp:142-197 (hybrid)
 * Threading: a context and the graphs made with it belong to one host thread
 * at a time (the reference drives BBTc from the main thread, src/bbtc.cu:40-89);
 * the request server (bbtc_server_*) is safe to call from any thread.
 */
#ifndef BBTC_GPU_H_
#define BBTC_GPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bbtc_status {
  BBTC_OK = 0,
  BBTC_ERR_ARG = -1,         /* bad argument (null pointer, out-of-range value) */
  BBTC_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  BBTC_ERR_NOMEM = -3,       /* device or host allocation failed */
  BBTC_ERR_INPUT = -4,       /* the CSR or cut vector breaks the input contract */
  BBTC_ERR_TIMEOUT = -5,     /* a bounded device wait ran out */
  BBTC_ERR_NODEV = -6,       /* no usable CUDA device / wrong device index */
  BBTC_ERR_UNSUPPORTED = -7, /* valid request this build does not serve */
  BBTC_ERR_STATE = -8,       /* call out of order (e.g. polling an unknown request) */
  BBTC_ERR_CAPACITY = -9,    /* admission refused: over the HBM budget or slot limit */
  BBTC_ERR_LAYOUT = -10      /* bbtc_graph_validate found the device layout broken */
} bbtc_status;

typedef struct bbtc_ctx bbtc_ctx;
typedef struct bbtc_graph bbtc_graph;

/* Copy the calling thread's last error message (NUL-terminated, truncated). */
int bbtc_last_error(char* buf, size_t len);

/* Library version as major*10000 + minor*100 + patch. */
int bbtc_version(void);

/* Fault-injection hook for tests: the device allocation that follows `after`
 * more successful ones fails once, as if the device were out of memory (the
 * call that made it returns BBTC_ERR_NOMEM); after < 0 disarms.  *left (may
 * be NULL) receives the state before the call: -1 when nothing was armed or
 * the armed fault has fired, else the allocations it was still to let pass.
 * BBTC_FAIL_ALLOC=k in the environment arms it when the library loads.
 * Process-wide (all contexts and threads). */
int bbtc_debug_fail_alloc(int64_t after, int64_t* left);

/* Test hook for the bounded device waits: with polls > 0, the per-task
 * kernels of this context (BBTC_KERNEL_BITMAP / SEARCH) no longer issue their
 * shared-memory staging copies, and each staging wait gives up after `polls`
 * polls, as it would for a copy that never lands: the count is void and the
 * call returns BBTC_ERR_TIMEOUT, with nothing left in flight.  0 restores
 * normal staging.  No reference counterpart (it checks no wait or error). */
int bbtc_debug_stage_timeout(bbtc_ctx* ctx, uint32_t polls);

/* ---- context: device, stream, scratch ------------------------------------
 * Replaces BBTc's constructor GPU set-up and PrepareGpu
 * (src/triangle_counting/bb_tc.cpp:17-33, bb_tc_helper.cpp:53-73): one
 * stream, no per-stream global bitmap.  Only device 0..count-1 are valid;
 * the reference's multi-GPU striping (--ngpu > 1) is not served. */
int bbtc_ctx_create(int device, bbtc_ctx** out);
int bbtc_ctx_destroy(bbtc_ctx* ctx);
/* The cudaStream_t the context launches on (returned as void*). */
int bbtc_ctx_stream(bbtc_ctx* ctx, void** stream);
/* Number of SMs of the context's device. */
int bbtc_ctx_sm_count(bbtc_ctx* ctx, int* sms);
/* Host uploads of this context: an indptr or indices array of at most
 * max_bytes that lies wholly in one page-locked host allocation mapped into
 * the device's address space (cudaHostAlloc / cudaMallocHost memory, or
 * cudaHostRegister'd ranges) is read by a kernel over the host link instead
 * of being queued on the copy engines, where a small transfer waits behind
 * other streams' large ones.  Anything else is copied as usual.  0 (the
 * default) turns it off.  The server turns it on for small requests. */
int bbtc_ctx_set_zero_copy(bbtc_ctx* ctx, uint64_t max_bytes);

/* ---- graph: device-resident block CSR ------------------------------------
 * Replaces BlockCSR(cuts, x_adj, adj) + CSRtoBCSR (block_csr.cpp:35-42,
 * 288-376) and the lazy per-tile copies of CopyTileToGpu
 * (bb_tc_helper.cpp:75-110).  Input contract:
 *   - indptr[n+1], indices[m]: CSR with indptr[0] = 0, indptr[n] = m,
 *     non-decreasing; every row strictly increasing; every id < n.
 *     (The counting graph is the degree-ordered, oriented one; the count is
 *     the reference's task sum for any CSR that meets this contract.)
 *   - cuts[P+1]: cuts[0] = 0, non-decreasing, cuts[P] >= n (rows >= n are
 *     empty, like the phantom row the reference adds, utils.hpp:288); 1 <= P <= 64.
 * The library builds every tile's CSR and CSC on the device; segments start
 * 16-byte aligned.  The caller keeps its buffers. */
int bbtc_graph_upload(bbtc_ctx* ctx, uint32_t n, const uint32_t* indptr, const uint32_t* indices,
                      uint64_t m, const uint32_t* cuts, uint32_t P, bbtc_graph** out);
/* Same, with indptr / indices already in device memory of the context's
 * device (cuts stay on the host).  Nothing is copied from the host. */
int bbtc_graph_upload_device(bbtc_ctx* ctx, uint32_t n, const uint32_t* d_indptr,
                             const uint32_t* d_indices, uint64_t m, const uint32_t* cuts, uint32_t P,
                             bbtc_graph** out);
int bbtc_graph_free(bbtc_graph* g);

typedef struct bbtc_graph_info {
  uint32_t n;             /* rows (vertices) */
  uint32_t P;             /* number of parts (the reference's --ncut) */
  uint64_t m;             /* oriented edges, the reference's "Number of Edges" */
  uint64_t device_bytes;  /* device memory the graph holds */
  double layout_ms;       /* device time of the layout build */
  uint32_t zero_copy;     /* 1: the upload read the host CSR with a kernel (bbtc_ctx_set_zero_copy) */
  uint32_t reserved;
} bbtc_graph_info;
int bbtc_graph_info_get(const bbtc_graph* g, bbtc_graph_info* info);

/* Debug check of the device layout: copies every array of g back and checks
 * on the host what the counting kernels rely on -- the CSR contract; the
 * word-compressed rows expand to the rows; every tile's row pointers start
 * at 0, never decrease and end at its nnz; segments start on 16-byte
 * boundaries, stay inside their pools and do not overlap; tile rows are
 * strictly increasing, columns < the tile width, and together hold every
 * edge exactly once; tile statistics, the row index of every 32nd entry and
 * the reversed tiles' forward-edge records are right.  BBTC_ERR_LAYOUT with
 * the first broken rule in the message.  Costs about the graph's device
 * bytes in host memory; synchronises the context's stream. */
int bbtc_graph_validate(const bbtc_graph* g);

/* Per-tile statistics, row-major over the P x P grid (any pointer may be
 * NULL).  nnz / height are the reference's GetNNZ / GetHeight
 * (block_csr.cpp:88-92, 183-186); tile_deg = nnz / height is GetTileDeg
 * (block_csr.cpp:258-284).  max_deg = longest row of the tile. */
int bbtc_graph_tile_stats(const bbtc_graph* g, uint32_t* nnz, uint32_t* height, uint32_t* width,
                          float* tile_deg, uint32_t* max_deg);

/* ---- tasks ----------------------------------------------------------------
 * A task names three tiles by row-major id: ab = i*P+j, bc = j*P+k,
 * ac = i*P+k, i <= j <= k -- the entries of tasks::TaskList (tasks.hpp:7-17). */
typedef struct bbtc_task {
  uint32_t ab, bc, ac;
} bbtc_task;

/* Fill the P(P+1)(P+2)/6 tasks in TaskList order.  With out == NULL only
 * *ntasks is set; otherwise cap must hold them all. */
int bbtc_task_list(uint32_t P, bbtc_task* out, uint32_t cap, uint32_t* ntasks);
/* Sort by the reference weight nnz(ab) * max(tile_deg(bc), tile_deg(ac))
 * (tasks.hpp:19-34); descending != 0 gives the CUDA build's order.  Ties keep
 * list order (stable). */
int bbtc_sort_tasks(const bbtc_graph* g, bbtc_task* tasks, uint32_t ntasks, int descending);

/* ---- counting --------------------------------------------------------------- */
typedef enum bbtc_mode {
  BBTC_MODE_PERSISTENT = 0, /* one launch pulls every task's work units from a device queue */
  BBTC_MODE_PLAIN = 1       /* one launch per task, like NoOfTrianglesInGPU (bb_tc.cpp:76-115) */
} bbtc_mode;

typedef enum bbtc_kernel {
  BBTC_KERNEL_AUTO = 0,   /* persistent form over the whole task list (tasks == NULL, or every task
                             once in any order, as the reference's driver passes it): fused task rows; otherwise
                             per task: bitmap when the part fits the shared bitmap, else search */
  BBTC_KERNEL_BITMAP = 1, /* per task: pivot row of bc as a shared-memory bitmap, probes from ac */
  BBTC_KERNEL_SEARCH = 2, /* per task: pivot row of bc as a sorted shared-memory list, bisection probes */
  BBTC_KERNEL_MERGE = 3,  /* per task, the reference's row order: pivot = ac row of each ab row,
                             the bc rows it meets are searched against it */
  BBTC_KERNEL_FUSED = 4   /* task rows: the tasks (i, j, k >= j) sharing tile ab = (i, j) in one
                             pass (needs the whole task list: tasks == NULL, or every task once) */
} bbtc_kernel;

typedef struct bbtc_opts {
  int mode;                  /* bbtc_mode */
  int kernel;                /* bbtc_kernel */
  uint32_t bitmap_words;     /* shared bitmap / list words per warp: 0 = default (1024) */
  uint32_t warps_per_block;  /* 0 = default (8) */
  uint32_t unit_work;        /* target probes per work unit, 0 = default (256 task rows, 8192 tasks) */
  uint32_t blocks_per_sm;    /* persistent grid = SMs x this, 0 = occupancy limit */
  int use_cuda_graph;        /* replay the launch sequence through a captured CUDA graph */
  int sort_tasks;            /* when tasks == NULL: 1 = cost-sorted descending (default) */
  uint32_t occupancy;        /* persistent form: register budget for 4, 5, 6 or 8 blocks per SM (5: fused task rows only; 0: 6 for
                                fused task rows with a bitmap of at most 1024 words, else 4) */
} bbtc_opts;

void bbtc_opts_default(bbtc_opts* o);

/* Count triangles: the sum over tasks of sum_{r in ab} sum_{b in ab[r]} |ac[r] ∩ bc[b]|.
 * tasks == NULL counts the whole TaskList(P) (sorted per opts->sort_tasks).
 * border follows --border (utils.hpp:111-114, bbtc.cu:54-62): -1 = every task
 * on the GPU; b >= 0 = tasks [0, b) are queued first, then the rest; all on
 * the GPU (CPU workers beside it: bbtc_count_hybrid).  *out receives the
 * exact count.
 * Replaces BBTc::NoOfTriangles (bb_tc.cpp:200-252). */
int bbtc_count(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_task* tasks, uint32_t ntasks, int32_t border,
               const bbtc_opts* opts, uint64_t* out);

/* Enqueue the same count on the context's stream without waiting; the count
 * lands in device memory owned by the graph.  bbtc_count_wait synchronises the
 * stream and returns it.  Used to time the device path with stream events. */
int bbtc_count_async(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_task* tasks, uint32_t ntasks,
                     int32_t border, const bbtc_opts* opts);
int bbtc_count_wait(bbtc_ctx* ctx, bbtc_graph* g, uint64_t* out);

/* Launches of this library's kernels issued by the last count on g. */
int bbtc_last_launches(const bbtc_graph* g, uint32_t* launches);

/* ---- autotuner ------------------------------------------------------------
 * Times the count of g under every combination of the listed shared-buffer
 * sizes (the bitmap-vs-search threshold: a pivot row becomes a bitmap when its
 * id span fits, else a sorted list), warps per block and work-unit sizes, and
 * writes the fastest into *inout (mode and kernel are kept).  Every point must
 * give the same count, else BBTC_ERR_STATE.  NULL space = the default sweep.
 * No reference counterpart: the reference fixes its kernel choice by a width
 * test (bb_tc.cpp:98). */
typedef struct bbtc_tune_space {
  const uint32_t* bitmap_words;
  uint32_t n_bitmap_words;
  const uint32_t* warps_per_block;
  uint32_t n_warps_per_block;
  const uint32_t* unit_work;
  uint32_t n_unit_work;
  uint32_t repeats; /* timed counts per point, the median is kept (0 = 3) */
  const uint32_t* occupancy;
  uint32_t n_occupancy;
} bbtc_tune_space;
int bbtc_autotune(bbtc_ctx* ctx, bbtc_graph* g, const bbtc_tune_space* space, bbtc_opts* inout,
                  double* best_ms);

/* Count many graphs in one persistent launch: every graph's TaskList(P)
 * goes into one cost-sorted device queue, each graph gets its own u64.  outs[ng]. */
int bbtc_count_batch(bbtc_ctx* ctx, bbtc_graph* const* graphs, uint32_t ng, const bbtc_opts* opts,
                     uint64_t* outs);

/* ---- hybrid GPU + CPU execution ---------------------------------------------
 * BBTc::NoOfTriangles with CPU workers beside the GPU (bb_tc.cpp:142-252,
 * RunGpuKernels :142-181, RunCpuKernels :184-197; Separator from --border,
 * bbtc.cu:54-62).  The border gives the Separator: -1 (or a value past the
 * end) = every task on the GPU, -2 = half the list, b >= 0 = b.  Tasks
 * [0, Separator) run on the GPU only; the rest are shared: cpu_workers host
 * threads take them one at a time from the tail, while the GPU takes them
 * from the head in list order, a contiguous range per bbtc_count launch, and
 * stops at the first task a CPU worker holds.  Every task is counted once;
 * *out is the sum.  tasks == NULL = TaskList(P) sorted heaviest first, the
 * reference's CUDA driver order.  indptr / indices are the host CSR the graph
 * was uploaded from (CPU workers read it; it must stay unchanged during the
 * call; NULL is allowed when cpu_workers = 0).  CPU workers check the rows
 * (strictly increasing, ids < n) before any of them counts: BBTC_ERR_INPUT if
 * they break the contract.  With cpu_workers = 0 this is bbtc_count.  The
 * context's GPU is required either way.  stats may be NULL. */
typedef struct bbtc_hybrid_stats {
  uint32_t gpu_tasks;    /* tasks counted on the GPU */
  uint32_t cpu_tasks;    /* tasks counted by the CPU workers */
  uint32_t gpu_launches; /* bbtc_count calls made by the GPU side */
  uint32_t separator;    /* the Separator the border gave */
  uint64_t gpu_count;    /* the GPU tasks' sum */
  uint64_t cpu_count;    /* the CPU tasks' sum */
  double gpu_ms;         /* wall time of the GPU side */
  double cpu_ms;         /* wall time of the slowest CPU worker */
} bbtc_hybrid_stats;
int bbtc_count_hybrid(bbtc_ctx* ctx, bbtc_graph* g, const uint32_t* indptr, const uint32_t* indices,
                      const bbtc_task* tasks, uint32_t ntasks, int32_t border, uint32_t cpu_workers,
                      const bbtc_opts* opts, uint64_t* out, bbtc_hybrid_stats* stats);

/* ---- device-side input preparation ------------------------------------------
 * The reference prepares the counting graph on the host: symmetrise, drop
 * self-loops (include/utils/utils.hpp:172-250), relabel by ascending degree
 * and keep the upper triangle (SARMA csr_matrix.hpp:503-584).
 * bbtc_orient_device does it on the GPU for m_raw pairs already in device
 * memory (ids >= n and repeated pairs are dropped; degree ties go by id), and
 * returns a library-allocated oriented CSR that bbtc_graph_upload_device
 * takes; free it with bbtc_csr_dev_free.  bbtc_rmat_device fills d_src /
 * d_dst (edge_factor << scale entries each) with R-MAT pairs drawn from the
 * same counter-based stream as the host generator, so both give the same
 * graph for the same seed. */
typedef struct bbtc_csr_dev {
  uint32_t* indptr;  /* n + 1 */
  uint32_t* indices; /* m */
  uint32_t n;
  uint64_t m;
} bbtc_csr_dev;
int bbtc_rmat_device(bbtc_ctx* ctx, int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                     uint32_t* d_src, uint32_t* d_dst);
int bbtc_orient_device(bbtc_ctx* ctx, uint32_t n, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m_raw,
                       bbtc_csr_dev* out);
int bbtc_csr_dev_free(bbtc_ctx* ctx, bbtc_csr_dev* csr);

/* Cut vector (P + 1 entries, host memory) of a CSR in device memory: the
 * partitioner on the GPU.  Replaces the host-side SARMA call of the
 * reference (include/utils/utils.hpp:271-288) for graphs that live on the
 * device.  kind: 0 = uni, 1 = n1d, 2 = pal (seed: the pal sampling seed, the
 * reference passes 1091467301).  Gives the same cuts as the host library's
 * bbtcp_cuts on the same CSR.  Synchronises the context's stream. */
int bbtc_cuts_device(bbtc_ctx* ctx, int kind, uint32_t n, const uint32_t* d_indptr, const uint32_t* d_indices,
                     uint64_t m, uint32_t P, uint64_t seed, uint32_t* cuts);

/* ---- request server: continuous batching ----------------------------------
 * No counterpart in the reference (one graph per process).  Loader threads
 * build each submitted graph's device block CSR on their own streams,
 * admitting requests (smallest first, oldest first once they have waited
 * aging_ms) while their estimated device footprint fits hbm_budget; two
 * launch lanes (small graphs / large graphs) each count every ready graph of
 * their class in a single persistent launch (one u64 slot per graph),
 * publish the counts and free
 * the graphs.  Requests that arrive while a launch runs are loaded meanwhile
 * and join the next launch.  All server calls are thread-safe.  The caller's
 * indptr / indices must stay valid until the request finishes (pinned host
 * memory makes the upload asynchronous); cuts are copied. */
typedef struct bbtc_server bbtc_server;
typedef struct bbtc_server_opts {
  uint64_t hbm_budget;    /* device bytes admitted graphs may hold (0 = 150 GiB) */
  uint32_t max_batch;     /* graphs per launch (0 = 4096) */
  uint32_t max_requests;  /* requests held (queued, running or finished, not released) (0 = 2^20) */
  uint32_t loaders;       /* loader threads, each with its own stream (0 = 6) */
  uint32_t copy_engine_uploads; /* 1: small requests' CSRs always go through the copy engines; 0 (default):
                                   from page-locked host buffers they are read by a kernel
                                   (bbtc_ctx_set_zero_copy) */
  bbtc_opts count;        /* launch options of every batch */
  uint64_t small_edges;   /* graphs of at most this many edges use the high-priority lane (0 = 2^22) */
  uint32_t large_blocks_per_sm; /* persistent blocks per SM of the large lane (0 = 3) */
  uint32_t aging_ms;      /* a request waiting this long is loaded before smaller ones (default 50) */
  uint64_t pool_bytes;    /* the device memory pool is grown to this size at creation, so loads never
                             wait for it to grow (0 = 1.1 x hbm_budget; at most the free memory less 8 GiB) */
  uint32_t large_layout_blocks_per_sm; /* grid cap of the large requests' layout kernels, blocks of 256 threads per
                                          SM (0 = 2), so that small requests' kernels find room on every SM */
  uint32_t max_large_loads; /* large requests uploaded and laid out at once, at most (default 2; 0 = no limit) */
  uint32_t small_sms;       /* > 0: a partition of this many SMs (a multiple of 8; green contexts) runs the small
                               requests' loads and counts, the other SMs the large ones', so neither waits for
                               the other's blocks (0 = all SMs shared) */
  uint32_t small_aging_us;  /* a small request waiting this long (microseconds) is loaded before smaller ones
                               (0 = aging_ms) */
} bbtc_server_opts;
typedef struct bbtc_request_info {
  uint64_t count;     /* exact count once status == 1 */
  int32_t status;     /* 0 in flight, 1 done, < 0 failed with that bbtc_status */
  uint32_t batch;     /* graphs in the launch that counted it */
  uint64_t submit_ns; /* steady-clock time of bbtc_submit */
  uint64_t done_ns;   /* steady-clock time the count reached host memory */
  uint64_t load_ns;   /* a loader took the request (upload + layout start) */
  uint64_t ready_ns;  /* its layout was built */
  uint64_t launch_ns; /* the launch that counted it was issued */
} bbtc_request_info;
typedef struct bbtc_server_stats {
  uint64_t launches, counted, max_batch, pending, ready, device_bytes_in_use;
} bbtc_server_stats;
/* The server runs 2 x loaders + 2 streams.  Give each its own hardware work
 * queue: set CUDA_DEVICE_MAX_CONNECTIONS=32 in the environment before the
 * process first initialises CUDA (bbtc_server_create sets it when unset, which
 * helps only if no CUDA call came earlier).  With the default of 8, streams
 * share queues and a small request's launch can wait for a large count. */
void bbtc_server_opts_default(bbtc_server_opts* o);
int bbtc_server_create(int device, const bbtc_server_opts* opts, bbtc_server** out);
/* Finishes loads in progress and ready graphs; requests still queued fail with BBTC_ERR_STATE. */
int bbtc_server_destroy(bbtc_server* s);
int bbtc_submit(bbtc_server* s, uint32_t n, const uint32_t* indptr, const uint32_t* indices, uint64_t m,
                const uint32_t* cuts, uint32_t P, uint64_t* req_id);
int bbtc_poll(bbtc_server* s, uint64_t req_id, bbtc_request_info* info);
/* timeout_ms < 0 waits for ever; BBTC_ERR_TIMEOUT if the request is still in flight */
int bbtc_wait(bbtc_server* s, uint64_t req_id, int64_t timeout_ms, bbtc_request_info* info);
/* Forget a finished request (its id becomes unknown). */
int bbtc_release(bbtc_server* s, uint64_t req_id);
int bbtc_server_stats_get(bbtc_server* s, bbtc_server_stats* st);

/* ---- counting without allocation -------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory -- code running inside another framework's
 * device-memory manager that owns the device's memory and hands out only
 * slices of its own pool, processes held to a fixed device-memory quota, and
 * paths that must not pay the implicit device synchronisation of cudaMalloc /
 * cudaFree.  The caller passes a degree-ordered, oriented CSR that is already
 * in device memory of the current device (d_indptr[n+1], d_indices[m], rows
 * strictly increasing) and a host pointer for the count; the call allocates
 * nothing.  Its scratch (queue head, error word, total, one partial count per
 * 256 edges) is a file-scope device array of about 512 KiB that every GPU
 * loading the library holds until the process exits, so m is limited to
 * 16,777,216 oriented edges (larger m: BBTC_ERR_CAPACITY, nothing launched).
 * The first call on a device (with that device current) looks up the array's
 * device address and the kernel's launch shape, once.  All calls share the
 * array and it keeps the last call's contents: each call clears what must
 * start at zero, and calls that overlap on the GPU (on different streams or
 * threads) race -- serialise them.  Work is enqueued on `stream` (a
 * cudaStream_t, NULL = the legacy default stream) and the call is synchronous:
 * it waits for that stream before returning, so it must not be called while
 * the stream is being captured.  n == 0 with m > 0 is BBTC_ERR_ARG; a row
 * pointer or id out of bounds (indptr[n] < m included), or an unsorted row,
 * is reported as BBTC_ERR_INPUT without reading outside the caller's arrays
 * (indptr[n+1], indices[m]). */
int bbtc_count_csr_noalloc(const uint32_t* d_indptr, const uint32_t* d_indices, uint32_t n, uint64_t m,
                           uint64_t* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BBTC_GPU_H_ */

"""Python binding of the C ABI in include/bbtc_gpu.h (libbbtc.so).

The objects mirror the reference's driver sequence (src/bbtc.cu:28-89):

    st    = Graph.upload(ctx, csr, cuts)       # BlockCSR(cuts, x_adj, adj)
    tl    = st.task_list(sorted=True)          # tasks::TaskList + SortTasks
    bbtc  = BBTc(st, tl)                       # BBTc(&st, tasks, P)
    bbtc.Separator = -1                        # --border
    n     = bbtc.NoOfTriangles()               # exact u64 count

Every failing C call raises :class:`BBTcError` with the library's message.
There is no CPU path: without libbbtc.so or a B200 the calls fail.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib

c = ctypes

STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_NOMEM", -4: "ERR_INPUT", -5: "ERR_TIMEOUT",
          -6: "ERR_NODEV", -7: "ERR_UNSUPPORTED", -8: "ERR_STATE", -9: "ERR_CAPACITY",
          -10: "ERR_LAYOUT"}

MODE_PERSISTENT, MODE_PLAIN = 0, 1
KERNEL_AUTO, KERNEL_BITMAP, KERNEL_SEARCH, KERNEL_MERGE, KERNEL_FUSED = 0, 1, 2, 3, 4
KERNELS = {"auto": KERNEL_AUTO, "bitmap": KERNEL_BITMAP, "search": KERNEL_SEARCH, "merge": KERNEL_MERGE,
           "fused": KERNEL_FUSED}
MODES = {"persistent": MODE_PERSISTENT, "plain": MODE_PLAIN}


class BBTcError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.message = message


class Task(c.Structure):
    _fields_ = [("ab", c.c_uint32), ("bc", c.c_uint32), ("ac", c.c_uint32)]


class Opts(c.Structure):
    _fields_ = [("mode", c.c_int), ("kernel", c.c_int), ("bitmap_words", c.c_uint32),
                ("warps_per_block", c.c_uint32), ("unit_work", c.c_uint32), ("blocks_per_sm", c.c_uint32),
                ("use_cuda_graph", c.c_int), ("sort_tasks", c.c_int), ("occupancy", c.c_uint32)]


class GraphInfo(c.Structure):
    _fields_ = [("n", c.c_uint32), ("P", c.c_uint32), ("m", c.c_uint64), ("device_bytes", c.c_uint64),
                ("layout_ms", c.c_double), ("zero_copy", c.c_uint32), ("reserved", c.c_uint32)]


class HybridStats(c.Structure):
    _fields_ = [("gpu_tasks", c.c_uint32), ("cpu_tasks", c.c_uint32), ("gpu_launches", c.c_uint32),
                ("separator", c.c_uint32), ("gpu_count", c.c_uint64), ("cpu_count", c.c_uint64),
                ("gpu_ms", c.c_double), ("cpu_ms", c.c_double)]


TASK_DTYPE = np.dtype([("ab", np.uint32), ("bc", np.uint32), ("ac", np.uint32)])

_typed = False


def lib() -> ctypes.CDLL:
    global _typed
    L = _lib._load("libbbtc.so")
    if _typed:
        return L
    vp, u32, u64, i32 = c.c_void_p, c.c_uint32, c.c_uint64, c.c_int32
    sig = {
        "bbtc_last_error": [c.c_char_p, c.c_size_t],
        "bbtc_version": [],
        "bbtc_debug_fail_alloc": [c.c_int64, c.POINTER(c.c_int64)],
        "bbtc_debug_stage_timeout": [vp, u32],
        "bbtc_ctx_create": [c.c_int, c.POINTER(vp)],
        "bbtc_ctx_destroy": [vp],
        "bbtc_ctx_stream": [vp, c.POINTER(vp)],
        "bbtc_ctx_sm_count": [vp, c.POINTER(c.c_int)],
        "bbtc_ctx_set_zero_copy": [vp, u64],
        "bbtc_graph_upload": [vp, u32, vp, vp, u64, vp, u32, c.POINTER(vp)],
        "bbtc_graph_upload_device": [vp, u32, vp, vp, u64, vp, u32, c.POINTER(vp)],
        "bbtc_graph_free": [vp],
        "bbtc_graph_info_get": [vp, c.POINTER(GraphInfo)],
        "bbtc_graph_tile_stats": [vp, vp, vp, vp, vp, vp],
        "bbtc_graph_validate": [vp],
        "bbtc_task_list": [u32, vp, u32, c.POINTER(u32)],
        "bbtc_sort_tasks": [vp, vp, u32, c.c_int],
        "bbtc_count": [vp, vp, vp, u32, i32, c.POINTER(Opts), c.POINTER(u64)],
        "bbtc_count_async": [vp, vp, vp, u32, i32, c.POINTER(Opts)],
        "bbtc_count_wait": [vp, vp, c.POINTER(u64)],
        "bbtc_last_launches": [vp, c.POINTER(u32)],
        "bbtc_count_batch": [vp, vp, u32, c.POINTER(Opts), vp],
        "bbtc_count_hybrid": [vp, vp, vp, vp, vp, u32, i32, u32, c.POINTER(Opts), c.POINTER(u64),
                              c.POINTER(HybridStats)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = c.c_int
    L.bbtc_opts_default.argtypes = [c.POINTER(Opts)]
    L.bbtc_opts_default.restype = None
    _typed = True
    return L


def last_error() -> str:
    buf = c.create_string_buffer(1024)
    lib().bbtc_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def debug_fail_alloc(after: int) -> int:
    """Test hook: fail the device allocation that follows `after` more
    successful ones (after < 0 disarms).  Returns the previous state: -1 when
    nothing was armed or the armed fault has fired, else the allocations it
    was still to let pass."""
    left = c.c_int64()
    check(lib().bbtc_debug_fail_alloc(int(after), c.byref(left)))
    return left.value


def check(rc: int) -> None:
    if rc != 0:
        raise BBTcError(rc, last_error())


def options(mode: str | int = "persistent", kernel: str | int = "auto", bitmap_words: int = 0,
            warps_per_block: int = 0, unit_work: int = 0, blocks_per_sm: int = 0, cuda_graph: bool = True,
            sort_tasks: bool = True, occupancy: int = 0) -> Opts:
    o = Opts()
    lib().bbtc_opts_default(c.byref(o))
    o.mode = MODES[mode] if isinstance(mode, str) else int(mode)
    o.kernel = KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
    if bitmap_words:
        o.bitmap_words = bitmap_words
    if warps_per_block:
        o.warps_per_block = warps_per_block
    if unit_work:
        o.unit_work = unit_work
    o.blocks_per_sm = blocks_per_sm
    o.use_cuda_graph = 1 if cuda_graph else 0
    o.sort_tasks = 1 if sort_tasks else 0
    if occupancy:
        o.occupancy = occupancy
    return o


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


class Context:
    """A device + stream (bbtc_ctx)."""

    def __init__(self, device: int = 0):
        self._h = c.c_void_p()
        check(lib().bbtc_ctx_create(device, c.byref(self._h)))
        self.device = device

    @property
    def handle(self) -> c.c_void_p:
        if not self._h:
            raise BBTcError(-8, "context is closed")
        return self._h

    @property
    def stream(self) -> int:
        s = c.c_void_p()
        check(lib().bbtc_ctx_stream(self.handle, c.byref(s)))
        return s.value or 0

    def set_zero_copy(self, max_bytes: int) -> None:
        """Host arrays up to max_bytes in mapped page-locked memory are read by a
        kernel instead of the copy engines (0 turns it off)."""
        check(lib().bbtc_ctx_set_zero_copy(self.handle, int(max_bytes)))

    def debug_stage_timeout(self, polls: int) -> None:
        """Test hook: with polls > 0 the per-task kernels' staging copies are
        not issued and each staging wait gives up after `polls` polls, so a
        count that stages returns BBTC_ERR_TIMEOUT; 0 restores normal staging."""
        check(lib().bbtc_debug_stage_timeout(self.handle, int(polls)))

    @property
    def sm_count(self) -> int:
        v = c.c_int()
        check(lib().bbtc_ctx_sm_count(self.handle, c.byref(v)))
        return v.value

    def close(self) -> None:
        if self._h:
            lib().bbtc_ctx_destroy(self._h)
            self._h = c.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    """A device-resident block CSR (bbtc_graph): the reference's BlockCSR."""

    def __init__(self, ctx: Context, handle: c.c_void_p, n: int, m: int, cuts: np.ndarray):
        self.ctx = ctx
        self._h = handle
        self.n, self.m = n, m
        self.cuts = cuts
        self.P = len(cuts) - 1

    @classmethod
    def upload(cls, ctx: Context, n: int, indptr, indices, cuts) -> "Graph":
        """Host CSR -> device block CSR (bbtc_graph_upload)."""
        indptr, indices, cuts = _u32(indptr), _u32(indices), _u32(cuts)
        if indptr.shape[0] != n + 1:
            raise ValueError("indptr must have n+1 entries")
        h = c.c_void_p()
        check(lib().bbtc_graph_upload(ctx.handle, n, indptr.ctypes.data, indices.ctypes.data if indices.size else None,
                                      indices.size, cuts.ctypes.data, len(cuts) - 1, c.byref(h)))
        return cls(ctx, h, n, int(indices.size), cuts)

    @classmethod
    def upload_ptrs(cls, ctx: Context, n: int, indptr_ptr: int, indices_ptr: int, m: int, cuts) -> "Graph":
        """Host CSR given as raw host pointers (e.g. pinned buffers) -> device block CSR."""
        cuts = _u32(cuts)
        h = c.c_void_p()
        check(lib().bbtc_graph_upload(ctx.handle, n, indptr_ptr, indices_ptr, m, cuts.ctypes.data, len(cuts) - 1,
                                      c.byref(h)))
        return cls(ctx, h, n, m, cuts)

    @classmethod
    def upload_device(cls, ctx: Context, n: int, d_indptr: int, d_indices: int, m: int, cuts) -> "Graph":
        """Device CSR (raw device pointers) -> device block CSR."""
        cuts = _u32(cuts)
        h = c.c_void_p()
        check(lib().bbtc_graph_upload_device(ctx.handle, n, d_indptr, d_indices, m, cuts.ctypes.data,
                                             len(cuts) - 1, c.byref(h)))
        return cls(ctx, h, n, m, cuts)

    @classmethod
    def from_csr(cls, ctx: Context, csr, cuts) -> "Graph":
        return cls.upload(ctx, csr.n, csr.indptr, csr.indices, cuts)

    @property
    def handle(self) -> c.c_void_p:
        if not self._h:
            raise BBTcError(-8, "graph is freed")
        return self._h

    def info(self) -> GraphInfo:
        i = GraphInfo()
        check(lib().bbtc_graph_info_get(self.handle, c.byref(i)))
        return i

    def tile_stats(self) -> dict:
        T = self.P * self.P
        nnz = np.zeros(T, np.uint32)
        h = np.zeros(T, np.uint32)
        w = np.zeros(T, np.uint32)
        deg = np.zeros(T, np.float32)
        mx = np.zeros(T, np.uint32)
        check(lib().bbtc_graph_tile_stats(self.handle, nnz.ctypes.data, h.ctypes.data, w.ctypes.data,
                                          deg.ctypes.data, mx.ctypes.data))
        return dict(nnz=nnz, height=h, width=w, tile_deg=deg, max_deg=mx)

    def validate(self) -> None:
        """Copy the device layout back and check it on the host (BBTcError -10 if broken)."""
        check(lib().bbtc_graph_validate(self.handle))

    def task_list(self, sorted: bool = True, descending: bool = True) -> np.ndarray:
        t = task_list(self.P)
        if sorted:
            check(lib().bbtc_sort_tasks(self.handle, t.ctypes.data, len(t), 1 if descending else 0))
        return t

    def count(self, tasks: np.ndarray | None = None, border: int = -1, opts: Opts | None = None) -> int:
        out = c.c_uint64()
        tp, nt = _tasks_arg(tasks)
        check(lib().bbtc_count(self.ctx.handle, self.handle, tp, nt, border, c.byref(opts) if opts else None,
                               c.byref(out)))
        return out.value

    def count_hybrid(self, indptr, indices, tasks: np.ndarray | None = None, border: int = 0, cpu_workers: int = 1,
                     opts: Opts | None = None) -> tuple[int, dict]:
        """The count with CPU workers beside the GPU (bb_tc.cpp:142-252):
        tasks [0, Separator) on the GPU, the rest shared -- CPU workers from
        the tail, the GPU from the head.  indptr / indices: the host CSR this
        graph was uploaded from.  Returns (count, stats)."""
        ip = _u32(indptr)
        ix = _u32(indices) if len(indices) else np.zeros(1, np.uint32)
        out = c.c_uint64()
        st = HybridStats()
        tp, nt = _tasks_arg(tasks)
        check(lib().bbtc_count_hybrid(self.ctx.handle, self.handle, ip.ctypes.data, ix.ctypes.data, tp, nt, border,
                                      cpu_workers, c.byref(opts) if opts else None, c.byref(out), c.byref(st)))
        return out.value, {f: getattr(st, f) for f, _ in HybridStats._fields_}

    def count_async(self, tasks: np.ndarray | None = None, border: int = -1, opts: Opts | None = None) -> None:
        tp, nt = _tasks_arg(tasks)
        check(lib().bbtc_count_async(self.ctx.handle, self.handle, tp, nt, border, c.byref(opts) if opts else None))

    def count_wait(self) -> int:
        out = c.c_uint64()
        check(lib().bbtc_count_wait(self.ctx.handle, self.handle, c.byref(out)))
        return out.value

    def last_launches(self) -> int:
        v = c.c_uint32()
        check(lib().bbtc_last_launches(self.handle, c.byref(v)))
        return v.value

    def free(self) -> None:
        if self._h:
            lib().bbtc_graph_free(self._h)
            self._h = c.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _tasks_arg(tasks):
    if tasks is None:
        return None, 0
    t = np.ascontiguousarray(tasks, dtype=TASK_DTYPE)
    return t.ctypes.data, len(t)


def task_list(P: int) -> np.ndarray:
    """tasks::TaskList(P): (i <= j <= k) -> (ij, jk, ik) tile ids."""
    nt = c.c_uint32()
    check(lib().bbtc_task_list(P, None, 0, c.byref(nt)))
    t = np.zeros(nt.value, dtype=TASK_DTYPE)
    check(lib().bbtc_task_list(P, t.ctypes.data, nt.value, c.byref(nt)))
    return t


def count_batch(ctx: Context, graphs: list[Graph], opts: Opts | None = None) -> list[int]:
    arr = (c.c_void_p * len(graphs))(*[g.handle for g in graphs])
    outs = np.zeros(len(graphs), dtype=np.uint64)
    check(lib().bbtc_count_batch(ctx.handle, arr, len(graphs), c.byref(opts) if opts else None,
                                 outs.ctypes.data))
    return [int(x) for x in outs]


class BBTc:
    """The reference's driver object (include/triangle_counting/bb_tc.h:28-218)
    over the device layout: same method names.  By default every task runs on
    the GPU; SetCpuWorkers(k, indptr, indices) adds k CPU workers that take
    tasks past the Separator from the tail, as the reference's OpenMP workers
    do (bb_tc.cpp:184-197)."""

    def __init__(self, st: Graph, tasks: np.ndarray | None = None, P: int | None = None):
        if P is not None and P != st.P:
            raise ValueError("P does not match the graph's cut vector")
        self.st = st
        self.tasks = st.task_list(sorted=True) if tasks is None else np.ascontiguousarray(tasks, TASK_DTYPE)
        self.Separator = -1
        self.opts = options()
        self._ngpu = 1
        self._cpu = 0
        self._host = None
        self.last_stats: dict | None = None

    def SetCpuWorkers(self, k: int, indptr=None, indices=None) -> None:
        """k CPU workers beside the GPU; they read the host CSR the graph was uploaded from."""
        if k < 0:
            raise BBTcError(-1, "the number of CPU workers must be >= 0")
        if k > 0 and (indptr is None or indices is None):
            raise BBTcError(-1, "CPU workers need the host CSR (indptr, indices)")
        self._cpu = k
        self._host = (_u32(indptr), _u32(indices)) if k > 0 else None

    # InitFlags / ResetFlags / PrepareGpu / CopyTilesToGpu have nothing to do:
    # the queue lives on the device and the tiles are resident after upload.
    def InitFlags(self) -> None:
        pass

    def ResetFlags(self) -> None:
        pass

    def PrepareGpu(self) -> None:
        pass

    def CopyTilesToGpu(self) -> None:
        pass

    def SetNGPU(self, n: int) -> None:
        if n != 1:
            raise BBTcError(-7, "only one GPU is served (--ngpu 1)")
        self._ngpu = n

    def GetNGPU(self) -> int:
        return self._ngpu

    def NoOfTriangles(self) -> int:
        if self._cpu > 0:
            sep = -1 if self.Separator is None else int(self.Separator)
            count, self.last_stats = self.st.count_hybrid(self._host[0], self._host[1], self.tasks,
                                                          sep if sep >= -2 else -1, self._cpu, self.opts)
            return count
        border = -1 if self.Separator is None or self.Separator < 0 or self.Separator >= len(self.tasks) \
            else int(self.Separator)
        return self.st.count(self.tasks, border, self.opts)

    def CleanUp(self) -> None:
        self.st.free()


# ---- request server (continuous batching) ----------------------------------
class ServerOpts(c.Structure):
    _fields_ = [("hbm_budget", c.c_uint64), ("max_batch", c.c_uint32), ("max_requests", c.c_uint32),
                ("loaders", c.c_uint32), ("copy_engine_uploads", c.c_uint32), ("count", Opts),
                ("small_edges", c.c_uint64), ("large_blocks_per_sm", c.c_uint32), ("aging_ms", c.c_uint32),
                ("pool_bytes", c.c_uint64), ("large_layout_blocks_per_sm", c.c_uint32),
                ("max_large_loads", c.c_uint32), ("small_sms", c.c_uint32), ("small_aging_us", c.c_uint32)]


class RequestInfo(c.Structure):
    _fields_ = [("count", c.c_uint64), ("status", c.c_int32), ("batch", c.c_uint32), ("submit_ns", c.c_uint64),
                ("done_ns", c.c_uint64), ("load_ns", c.c_uint64), ("ready_ns", c.c_uint64),
                ("launch_ns", c.c_uint64)]


class ServerStats(c.Structure):
    _fields_ = [("launches", c.c_uint64), ("counted", c.c_uint64), ("max_batch", c.c_uint64),
                ("pending", c.c_uint64), ("ready", c.c_uint64), ("device_bytes_in_use", c.c_uint64)]


def _server_lib():
    L = lib()
    if getattr(L, "_server_typed", False):
        return L
    vp = c.c_void_p
    L.bbtc_server_opts_default.argtypes = [c.POINTER(ServerOpts)]
    L.bbtc_server_opts_default.restype = None
    for name, args in {
        "bbtc_server_create": [c.c_int, c.POINTER(ServerOpts), c.POINTER(vp)],
        "bbtc_server_destroy": [vp],
        "bbtc_submit": [vp, c.c_uint32, vp, vp, c.c_uint64, vp, c.c_uint32, c.POINTER(c.c_uint64)],
        "bbtc_poll": [vp, c.c_uint64, c.POINTER(RequestInfo)],
        "bbtc_wait": [vp, c.c_uint64, c.c_int64, c.POINTER(RequestInfo)],
        "bbtc_release": [vp, c.c_uint64],
        "bbtc_server_stats_get": [vp, c.POINTER(ServerStats)],
    }.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = c.c_int
    L._server_typed = True
    return L


class Server:
    """Continuous-batching count server (bbtc_server_*).  The host CSR arrays
    of a request are kept referenced here until the request is released."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_batch: int = 0, loaders: int = 0,
                 opts: Opts | None = None, small_edges: int = 0, large_blocks_per_sm: int = 0,
                 aging_ms: int | None = None, pool_bytes: int = 0, copy_engine_uploads: bool = False,
                 large_layout_blocks_per_sm: int = 0, max_large_loads: int | None = None, small_sms: int | None = None,
                 small_aging_us: int | None = None):
        L = _server_lib()
        so = ServerOpts()
        L.bbtc_server_opts_default(c.byref(so))
        if hbm_budget:
            so.hbm_budget = hbm_budget
        if max_batch:
            so.max_batch = max_batch
        if loaders:
            so.loaders = loaders
        if opts is not None:
            so.count = opts
        if small_edges:
            so.small_edges = small_edges
        if large_blocks_per_sm:
            so.large_blocks_per_sm = large_blocks_per_sm
        if aging_ms is not None:
            so.aging_ms = aging_ms
        if pool_bytes:
            so.pool_bytes = pool_bytes
        if large_layout_blocks_per_sm:
            so.large_layout_blocks_per_sm = large_layout_blocks_per_sm
        if max_large_loads is not None:
            so.max_large_loads = max_large_loads
        if small_sms is not None:
            so.small_sms = small_sms
        if small_aging_us is not None:
            so.small_aging_us = small_aging_us
        so.copy_engine_uploads = 1 if copy_engine_uploads else 0
        self._h = c.c_void_p()
        check(L.bbtc_server_create(device, c.byref(so), c.byref(self._h)))
        self._keep: dict[int, tuple] = {}

    def submit(self, n: int, indptr, indices, cuts) -> int:
        indptr, indices, cuts = _u32(indptr), _u32(indices), _u32(cuts)
        rid = c.c_uint64()
        check(_server_lib().bbtc_submit(self._h, n, indptr.ctypes.data,
                                        indices.ctypes.data if indices.size else None, indices.size,
                                        cuts.ctypes.data, len(cuts) - 1, c.byref(rid)))
        self._keep[rid.value] = (indptr, indices)
        return rid.value

    def submit_csr(self, csr, cuts) -> int:
        return self.submit(csr.n, csr.indptr, csr.indices, cuts)

    def poll(self, rid: int) -> RequestInfo:
        info = RequestInfo()
        check(_server_lib().bbtc_poll(self._h, rid, c.byref(info)))
        return info

    def wait(self, rid: int, timeout_ms: int = -1) -> RequestInfo:
        info = RequestInfo()
        check(_server_lib().bbtc_wait(self._h, rid, timeout_ms, c.byref(info)))
        return info

    def release(self, rid: int) -> None:
        check(_server_lib().bbtc_release(self._h, rid))
        self._keep.pop(rid, None)

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(_server_lib().bbtc_server_stats_get(self._h, c.byref(st)))
        return st

    def close(self) -> None:
        if self._h:
            _server_lib().bbtc_server_destroy(self._h)
            self._h = c.c_void_p()
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- device-side input preparation -------------------------------------------
class CsrDev(c.Structure):
    _fields_ = [("indptr", c.c_void_p), ("indices", c.c_void_p), ("n", c.c_uint32), ("m", c.c_uint64)]


def _prep_lib():
    L = lib()
    if getattr(L, "_prep_typed", False):
        return L
    vp = c.c_void_p
    for name, args in {
        "bbtc_rmat_device": [vp, c.c_int, c.c_int, c.c_double, c.c_double, c.c_double, c.c_uint64, vp, vp],
        "bbtc_orient_device": [vp, c.c_uint32, vp, vp, c.c_uint64, c.POINTER(CsrDev)],
        "bbtc_csr_dev_free": [vp, c.POINTER(CsrDev)],
        "bbtc_cuts_device": [vp, c.c_int, c.c_uint32, vp, vp, c.c_uint64, c.c_uint32, c.c_uint64, vp],
    }.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = c.c_int
    L._prep_typed = True
    return L


def rmat_device(ctx: Context, scale: int, edge_factor: int, d_src: int, d_dst: int, seed: int,
                a: float = 0.57, b: float = 0.19, cc: float = 0.19) -> None:
    """Fill device buffers (edge_factor << scale entries each) with R-MAT pairs."""
    check(_prep_lib().bbtc_rmat_device(ctx.handle, scale, edge_factor, a, b, cc, seed, d_src, d_dst))


def cuts_device(ctx: Context, kind: str | int, n: int, d_indptr: int, d_indices: int, m: int, P: int,
                seed: int = 1091467301) -> np.ndarray:
    """Cut vector of a device CSR computed on the GPU (bbtc_cuts_device): the
    same cuts as graphs.cuts on the same CSR.  kind: "uni", "n1d" or "pal"."""
    k = {"uni": 0, "n1d": 1, "pal": 2}[kind] if isinstance(kind, str) else int(kind)
    out = np.zeros(P + 1, dtype=np.uint32)
    check(_prep_lib().bbtc_cuts_device(ctx.handle, k, n, d_indptr, d_indices, m, P, seed, out.ctypes.data))
    return out


class DeviceCSR:
    """An oriented CSR built on the device by bbtc_orient_device."""

    def __init__(self, ctx: Context, n: int, d_src: int, d_dst: int, m_raw: int):
        self.ctx = ctx
        self._c = CsrDev()
        check(_prep_lib().bbtc_orient_device(ctx.handle, n, d_src, d_dst, m_raw, c.byref(self._c)))

    @property
    def n(self) -> int:
        return self._c.n

    @property
    def m(self) -> int:
        return self._c.m

    @property
    def indptr_ptr(self) -> int:
        return self._c.indptr

    @property
    def indices_ptr(self) -> int:
        return self._c.indices

    def graph(self, cuts) -> Graph:
        return Graph.upload_device(self.ctx, self.n, self.indptr_ptr, self.indices_ptr, self.m, cuts)

    def cuts(self, P: int, kind: str = "pal", seed: int = 1091467301) -> np.ndarray:
        """Cut vector computed on the GPU (bbtc_cuts_device)."""
        return cuts_device(self.ctx, kind, self.n, self.indptr_ptr, self.indices_ptr, self.m, P, seed)

    def free(self) -> None:
        if self._c.indptr:
            _prep_lib().bbtc_csr_dev_free(self.ctx.handle, c.byref(self._c))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

"""bbtc_b200 -- exact triangle counting over a 2D-partitioned block CSR on B200.

The counting path is libbbtc.so (CUDA, sm_100a) behind the C ABI in
include/bbtc_gpu.h; this package binds it (``core``), generates seeded input
graphs and cut vectors (``graphs``, host library libbbtc_host.so) and builds
everything in-tree (``build``).
"""
from .core import (BBTc, BBTcError, Context, Graph, KERNELS, MODES, Opts, Server, count_batch, options,  # noqa: F401
                   task_list)

__all__ = ["BBTc", "BBTcError", "Context", "Graph", "KERNELS", "MODES", "Opts", "Server", "count_batch", "options",
           "task_list"]

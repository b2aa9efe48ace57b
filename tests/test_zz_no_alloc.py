"""bbtc_count_csr_noalloc: the count for callers that cannot allocate device
memory (a framework that owns the device's memory, a fixed memory quota, or a
path that must not synchronise on cudaMalloc / cudaFree).  The caller brings a
device-resident CSR; the library's only scratch is a fixed static device array.
The count must equal the regular entry point's, call after call (the array
keeps the previous call's contents).  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from bbtc_b200 import Context, Graph, core, graphs

pytestmark = pytest.mark.gpu


def _noalloc():
    f = core.lib().bbtc_count_csr_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64,
                  ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _on_device(torch, g):
    ip = torch.from_numpy(g.indptr.view(np.int32)).cuda()
    ix = torch.from_numpy(g.indices.view(np.int32)).cuda()
    torch.cuda.synchronize()
    return ip, ix


def test_noalloc_matches_regular_count():
    torch = pytest.importorskip("torch")
    f = _noalloc()
    big = graphs.rmat(14, 16, seed=7)
    small = graphs.rgg(1 << 12, seed=8)
    with Context(0) as ctx:
        want = {}
        for g in (big, small):
            st = Graph.from_csr(ctx, g, graphs.cuts(g, 8, "pal"))
            want[g.name] = st.count()
            st.free()
    stream = torch.cuda.current_stream().cuda_stream
    dev = {g.name: _on_device(torch, g) for g in (big, small)}
    out = ctypes.c_uint64()
    # two calls in a row on the same graph, then another graph, then the first again
    for g in (big, big, small, big):
        ip, ix = dev[g.name]
        out.value = 0
        rc = f(ip.data_ptr(), ix.data_ptr(), g.n, g.m, ctypes.byref(out), stream)
        assert rc == 0, core.last_error()
        assert out.value == want[g.name], g.name
    assert want[big.name] > 0 and want[small.name] > 0


def test_noalloc_rejects_beyond_limit():
    torch = pytest.importorskip("torch")
    f = _noalloc()
    g = graphs.rmat(8, 8, seed=1)
    ip, ix = _on_device(torch, g)
    out = ctypes.c_uint64(123)
    rc = f(ip.data_ptr(), ix.data_ptr(), g.n, (1 << 24) + 1, ctypes.byref(out), None)
    assert rc == -9 and "16777216" in core.last_error()
    assert out.value == 123

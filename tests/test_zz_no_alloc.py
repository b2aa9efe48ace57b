"""bbtc_count_csr_noalloc: the count for callers that cannot allocate device
memory (a framework that owns the device's memory, a fixed memory quota, or a
path that must not synchronise on cudaMalloc / cudaFree).  The caller brings a
device-resident CSR; the library's only scratch is a fixed static device array.
The count must equal the oracle's and the regular entry point's, call after
call (the array keeps the previous call's contents).  This file is collected
last on purpose.
"""
import ctypes

import numpy as np
import pytest

import oracle
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
            cuts = graphs.cuts(g, 8, "pal")
            st = Graph.from_csr(ctx, g, cuts)
            want[g.name] = st.count()
            st.free()
            assert want[g.name] == oracle.count(g.n, g.indptr, g.indices, cuts)
            assert want[g.name] == oracle.count(g.n, g.indptr, g.indices, np.array([0, g.n], np.uint32))
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


def test_noalloc_malformed_inputs_are_refused():
    """Malformed CSRs inside allocations large enough for any stray read:
    each is refused with BBTC_ERR_INPUT (or BBTC_ERR_ARG for n == 0 with
    m > 0), and the next call counts right."""
    torch = pytest.importorskip("torch")
    f = _noalloc()
    g = graphs.rmat(10, 16, seed=3)
    want = oracle.count(g.n, g.indptr, g.indices, np.array([0, g.n], np.uint32))
    pad = 64

    def dev(a):
        t = torch.zeros(a.size + pad, dtype=torch.int32, device="cuda")
        t[:a.size] = torch.from_numpy(a.astype(np.uint32).view(np.int32))
        return t

    cases = []
    # m beyond indptr[n]: the padded indptr and indices hold zeros past the ends
    cases.append((g.indptr, g.indices, g.n, g.m + 40))
    # a row not in increasing order
    bad = g.indices.copy()
    u = int(np.argmax(np.diff(g.indptr.astype(np.int64)) >= 2))
    bad[g.indptr[u]], bad[g.indptr[u] + 1] = bad[g.indptr[u] + 1], bad[g.indptr[u]]
    cases.append((g.indptr, bad, g.n, g.m))
    # an id >= n
    big = g.indices.copy()
    big[g.m // 2] = g.n + 7
    cases.append((g.indptr, big, g.n, g.m))
    out = ctypes.c_uint64()
    for ip, ix, n, m in cases:
        dip, dix = dev(ip), dev(ix)
        torch.cuda.synchronize()
        out.value = 77
        rc = f(dip.data_ptr(), dix.data_ptr(), n, m, ctypes.byref(out), None)
        assert rc == -4, (rc, core.last_error())
        assert out.value == 77
    dip, dix = dev(g.indptr), dev(g.indices)
    torch.cuda.synchronize()
    assert f(dip.data_ptr(), dix.data_ptr(), 0, 5, ctypes.byref(out), None) == -1
    for _ in range(2):
        assert f(dip.data_ptr(), dix.data_ptr(), g.n, g.m, ctypes.byref(out), None) == 0, core.last_error()
        assert out.value == want

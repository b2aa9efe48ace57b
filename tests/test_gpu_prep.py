"""Device-side preparation equals the host pipeline bit for bit."""
import numpy as np
import pytest

import oracle
from bbtc_b200 import core, graphs

pytestmark = pytest.mark.gpu


class _DeviceView:
    """A zero-copy view of library-owned device memory for torch.as_tensor."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False), "version": 3}


def device_u32(torch, ptr, n):
    return torch.as_tensor(_DeviceView(ptr, n), device="cuda").cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("scale,ef,seed", [(8, 8, 1), (12, 16, 2), (16, 16, 1)])
def test_device_rmat_and_orient_equal_host(ctx, scale, ef, seed):
    torch = pytest.importorskip("torch")
    host = graphs.rmat(scale, ef, seed=seed)
    m_raw = ef << scale
    src = torch.empty(m_raw, dtype=torch.int32, device="cuda")
    dst = torch.empty(m_raw, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    core.rmat_device(ctx, scale, ef, src.data_ptr(), dst.data_ptr(), seed)
    dev = core.DeviceCSR(ctx, 1 << scale, src.data_ptr(), dst.data_ptr(), m_raw)
    assert dev.n == host.n and dev.m == host.m
    torch.cuda.synchronize()
    assert np.array_equal(device_u32(torch, dev.indptr_ptr, dev.n + 1), host.indptr)
    assert np.array_equal(device_u32(torch, dev.indices_ptr, dev.m), host.indices)
    cuts = graphs.cuts(host, 8, "uni")
    g = dev.graph(cuts)
    assert g.count() == oracle.count(host.n, host.indptr, host.indices, cuts)
    g.free()
    dev.free()


def test_orient_device_cleans_pairs(ctx):
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(3)
    n = 3000
    src = rng.integers(0, n, size=40000).astype(np.uint32)
    dst = rng.integers(0, n, size=40000).astype(np.uint32)
    src[:100] = dst[:100]  # self-loops
    src = np.concatenate([src, dst[:500], [n + 5]]).astype(np.uint32)  # reversed repeats, an id >= n
    dst = np.concatenate([dst, src[:500], [1]]).astype(np.uint32)
    host = graphs.from_pairs(n, src[:-1], dst[:-1])
    s = torch.from_numpy(src.view(np.int32)).cuda()
    d = torch.from_numpy(dst.view(np.int32)).cuda()
    torch.cuda.synchronize()
    dev = core.DeviceCSR(ctx, n, s.data_ptr(), d.data_ptr(), len(src))
    assert dev.m == host.m
    cuts = graphs.cuts(host, 5, "uni")
    g = dev.graph(cuts)
    assert g.count() == oracle.count(host.n, host.indptr, host.indices, cuts)
    g.free()
    dev.free()


@pytest.mark.parametrize("make", [lambda: graphs.rmat(8, 8, seed=1), lambda: graphs.rmat(16, 16, seed=2),
                                  lambda: graphs.rgg(1 << 14, seed=4),
                                  lambda: graphs.chung_lu(1 << 15, seed=5, max_deg=3000)])
def test_cuts_on_device_equal_host(ctx, make):
    """bbtc_cuts_device (the partitioner on the GPU) gives the host partitioners'
    cuts on the same CSR, for every kind and several stripe counts."""
    torch = pytest.importorskip("torch")
    g = make()
    ip = torch.from_numpy(g.indptr.view(np.int32)).cuda()
    ix = torch.from_numpy(g.indices.view(np.int32)).cuda()
    torch.cuda.synchronize()
    for kind in ("uni", "n1d", "pal"):
        for P in (1, 2, 5, 16, 64):
            got = core.cuts_device(ctx, kind, g.n, ip.data_ptr(), ix.data_ptr(), g.m, P)
            want = graphs.cuts(g, P, kind)
            assert np.array_equal(got, want), (kind, P, got, want)

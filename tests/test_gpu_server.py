"""Request server (continuous batching) and autotuner, on the GPU."""
import threading

import numpy as np
import pytest

import oracle
from bbtc_b200 import BBTcError, Graph, Server, autotune, graphs, options

pytestmark = pytest.mark.gpu


def mix():
    gs = [graphs.rmat(s, 8 + 4 * (s % 3), seed=300 + s) for s in (9, 10, 11, 12, 13, 14)]
    gs.append(graphs.rgg(1 << 12, seed=5))
    gs.append(graphs.chung_lu(1 << 13, seed=6, max_deg=400))
    return gs


def test_results_same_alone_and_in_the_mix(ctx):
    gs = mix()
    cuts = [graphs.cuts(g, 3 + i, "pal" if i % 2 else "uni") for i, g in enumerate(gs)]
    alone = []
    for g, c in zip(gs, cuts):
        st = Graph.from_csr(ctx, g, c)
        alone.append(st.count())
        st.free()
        assert alone[-1] == oracle.count(g.n, g.indptr, g.indices, c)
    order = [i for _ in range(4) for i in range(len(gs))]
    np.random.default_rng(1).shuffle(order)
    got = {}
    lock = threading.Lock()
    with Server(0, loaders=3) as srv:
        def client(part):
            for i in part:
                rid = srv.submit_csr(gs[i], cuts[i])
                with lock:
                    got[rid] = i
        ts = [threading.Thread(target=client, args=(order[k::4],)) for k in range(4)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        batched = 0
        for rid, i in got.items():
            info = srv.wait(rid, 60000)
            assert info.status == 1, info.status
            assert info.count == alone[i], (gs[i].name, info.count, alone[i])
            assert info.done_ns >= info.submit_ns
            batched += info.batch > 1
            srv.release(rid)
        st = srv.stats()
        assert st.counted == len(order) and st.launches >= 1 and st.pending == 0
    assert len(got) == len(order)


def test_admission_budget():
    small = graphs.rmat(9, 16, seed=7)
    big = graphs.rmat(18, 16, seed=8)  # about 3.6M edges: > 100 MB of layout
    cs, cb = graphs.cuts(small, 4, "uni"), graphs.cuts(big, 8, "uni")
    want_small = oracle.count(small.n, small.indptr, small.indices, cs)
    # a budget that holds the small graph (about 17 MB estimated) but never the big one
    with Server(0, hbm_budget=40 << 20) as srv:
        a = srv.submit_csr(small, cs)
        b = srv.submit_csr(big, cb)
        c = srv.submit_csr(small, cs)
        assert srv.wait(a, 60000).count == want_small
        assert srv.wait(b, 60000).status == -9  # BBTC_ERR_CAPACITY
        assert srv.wait(c, 60000).count == want_small


def test_server_errors():
    with Server(0) as srv:
        with pytest.raises(BBTcError):
            srv.poll(12345)
        bad = srv.submit(3, np.array([0, 2, 2, 2], np.uint32), np.array([2, 1], np.uint32), np.array([0, 3], np.uint32))
        assert srv.wait(bad, 60000).status == -4  # BBTC_ERR_INPUT: unsorted row
        g = graphs.rmat(9, 8, seed=3)
        ok = srv.submit_csr(g, graphs.cuts(g, 2, "uni"))
        assert srv.wait(ok, 60000).status == 1


def test_autotune_sweep_and_cache(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("BBTC_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    g = graphs.rmat(14, 16, seed=9)
    cuts = graphs.cuts(g, 8, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    try:
        o, ms = autotune.tune(st, bitmap_words=[256, 1024], warps_per_block=[4, 8], unit_work=[2048, 8192])
        assert ms is not None and ms > 0
        assert o.bitmap_words in (256, 1024) and o.warps_per_block in (4, 8)
        assert st.count(opts=o) == want
        o2, ms2 = autotune.tune(st)  # cache hit
        assert ms2 is None and o2.bitmap_words == o.bitmap_words and o2.unit_work == o.unit_work
    finally:
        st.free()


def _pinned(keep):
    import torch

    def pin(a):
        t = torch.empty(max(1, a.size), dtype=torch.int32, pin_memory=True)
        t.numpy()[:a.size] = a.view(np.int32)
        keep.append(t)
        return t.numpy()[:a.size].view(np.uint32)
    return pin


def test_pinned_requests_counted_right():
    """Small requests in page-locked buffers are read by a kernel (no copy
    engine); large ones, and the same graphs from pageable memory, are copied."""
    gs = mix()
    cuts = [graphs.cuts(g, 4 + i % 5, "uni") for i, g in enumerate(gs)]
    want = [oracle.count(g.n, g.indptr, g.indices, c) for g, c in zip(gs, cuts)]
    keep = []
    pin = _pinned(keep)
    pinned = [(pin(g.indptr), pin(g.indices)) for g in gs]
    for small_edges in (0, 1 << 12):  # default split, and most graphs on the large (copied) lane
        with Server(0, loaders=2, small_edges=small_edges) as srv:
            ids = []
            for rep in range(3):
                for i, g in enumerate(gs):
                    ip, ix = pinned[i] if rep != 1 else (g.indptr, g.indices)
                    ids.append((srv.submit(g.n, ip, ix, cuts[i]), i))
            for rid, i in ids:
                info = srv.wait(rid, 60000)
                assert info.status == 1 and info.count == want[i], (gs[i].name, info.status, info.count, want[i])
                srv.release(rid)


@pytest.mark.parametrize("small_sms", [8, 24])
def test_partitioned_server_counts(small_sms):
    """Small and large requests on separate SM partitions (green contexts):
    every count equals the oracle's, requests of both classes in flight at
    once, and a partition that leaves no SMs for the large requests is
    refused."""
    gs = mix() + [graphs.rmat(17, 16, seed=41)]
    small_edges = 1 << 16  # the s17 graph and the larger mix graphs take the large partition
    cuts = [graphs.cuts(g, 4 + i % 3, "uni") for i, g in enumerate(gs)]
    want = [oracle.count(g.n, g.indptr, g.indices, c) for g, c in zip(gs, cuts)]
    assert any(g.m > small_edges for g in gs) and any(g.m <= small_edges for g in gs)
    with Server(0, loaders=2, small_edges=small_edges, small_sms=small_sms) as srv:
        ids = [(srv.submit_csr(g, c), i) for _ in range(3) for i, (g, c) in enumerate(zip(gs, cuts))]
        for rid, i in ids:
            info = srv.wait(rid, 60000)
            assert info.status == 1 and info.count == want[i], (gs[i].name, info.status, info.count, want[i])
            srv.release(rid)
    with pytest.raises(BBTcError):
        Server(0, small_sms=100000)

"""Parity of the CUDA path (through the C ABI) with the oracle.

The oracle is the reference's CPU path: oracle.count (C restatement) and,
where built, oracle.ref_count (the reference's own sources).  Counts are
integers: every comparison is exact.
"""
import numpy as np
import pytest

import oracle
from bbtc_b200 import BBTc, BBTcError, Graph, count_batch, graphs, options

pytestmark = pytest.mark.gpu

KERNEL_MODES = [(k, m) for k in ("auto", "bitmap", "search", "merge", "fused") for m in ("persistent", "plain")]


def csr_from_edges(n, edges):
    src = np.array([e[0] for e in edges], dtype=np.uint32)
    dst = np.array([e[1] for e in edges], dtype=np.uint32)
    return graphs.from_pairs(n, src, dst)


def gpu_count(ctx, g, cuts, **kw):
    st = Graph.from_csr(ctx, g, cuts)
    try:
        return st.count(opts=options(**kw))
    finally:
        st.free()


@pytest.mark.parametrize("kernel,mode", KERNEL_MODES)
def test_rmat_small_all_paths(ctx, kernel, mode):
    g = graphs.rmat(12, 16, seed=1)
    for part, P in (("pal", 8), ("uni", 4), ("n1d", 16)):
        cuts = graphs.cuts(g, P, part)
        want = oracle.count(g.n, g.indptr, g.indices, cuts)
        assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode) == want, (part, P)


def test_config1_rmat16_pal8(ctx):
    """R-MAT scale 16, edge factor 16, seed 1, pal, ncut 8: the reference's
    CPU-runnable configuration, against the reference's own code."""
    g = graphs.rmat(16, 16, seed=1)
    cuts = graphs.cuts(g, 8, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    if oracle.ref_available():
        ref, _ = oracle.ref_count(g.n, g.indptr, g.indices, cuts)
        assert ref == want
    for kernel, mode in KERNEL_MODES:
        assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode) == want, (kernel, mode)


@pytest.mark.parametrize("bitmap_words,unit_work", [(32, 64), (64, 1), (256, 100000), (4096, 8192)])
def test_buffer_and_unit_sizes(ctx, bitmap_words, unit_work):
    """Small shared buffers force the list and global-memory pivot kinds; tiny
    units force many units per row."""
    g = graphs.rmat(13, 24, seed=5)
    cuts = graphs.cuts(g, 6, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    for kernel in ("auto", "search", "merge", "fused", "bitmap"):
        got = gpu_count(ctx, g, cuts, kernel=kernel, bitmap_words=bitmap_words, unit_work=unit_work)
        assert got == want, (kernel, bitmap_words, unit_work)


@pytest.mark.parametrize("warps", [1, 4, 8])
def test_warps_per_block(ctx, warps):
    g = graphs.rmat(11, 16, seed=9)
    cuts = graphs.cuts(g, 5, "uni")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    assert gpu_count(ctx, g, cuts, warps_per_block=warps) == want


def test_other_families(ctx):
    cases = [
        (graphs.rgg(1 << 14, seed=100), 8, "uni"),
        (graphs.chung_lu(1 << 15, seed=3, max_deg=2000), 16, "n1d"),
        (graphs.rmat(10, 32, seed=7), 4, "pal"),
    ]
    for g, P, part in cases:
        cuts = graphs.cuts(g, P, part)
        want = oracle.count(g.n, g.indptr, g.indices, cuts)
        assert want > 0
        for kernel, mode in KERNEL_MODES:
            assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode) == want, (g.name, kernel, mode)


def test_per_task_counts(ctx):
    """Every single task's sum equals the reference layout's task sum."""
    g = graphs.rmat(11, 16, seed=2)
    cuts = graphs.cuts(g, 5, "pal")
    st = Graph.from_csr(ctx, g, cuts)
    try:
        for t in st.task_list(sorted=False):
            want = oracle.task_count(g.n, g.indptr, g.indices, cuts, int(t["ab"]), int(t["bc"]), int(t["ac"]))
            one = np.array([t], dtype=t.dtype)
            for kernel in ("auto", "merge"):
                assert st.count(one, opts=options(kernel=kernel)) == want, (t, kernel)
        # the whole task list, in any order, runs as fused task rows
        total = oracle.count(g.n, g.indptr, g.indices, cuts)
        whole = st.task_list()
        for kernel in ("fused", "auto"):
            assert st.count(whole, opts=options(kernel=kernel)) == total, kernel
            assert st.count(whole[::-1].copy(), opts=options(kernel=kernel)) == total, kernel
        with pytest.raises(BBTcError):  # part of the list: fused task rows cannot run it
            st.count(whole[: len(whole) // 2].copy(), opts=options(kernel="fused"))
    finally:
        st.free()


def test_known_answers(ctx):
    n = 40
    kn = [(a, b) for a in range(n) for b in range(a + 1, n)]
    wheel = [(0, i) for i in range(1, 21)] + [(i, i % 20 + 1) for i in range(1, 21)]
    bip = [(a, b) for a in range(10) for b in range(10, 25)]
    star = [(0, i) for i in range(1, 50)]
    cases = [(n, kn, n * (n - 1) * (n - 2) // 6), (21, wheel, 20), (25, bip, 0), (50, star, 0)]
    for nv, edges, want in cases:
        g = csr_from_edges(nv, edges)
        for P in (1, 3, 7):
            cuts = graphs.cuts(g, P, "uni")
            for kernel, mode in KERNEL_MODES:
                assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode) == want, (nv, P, kernel, mode)


def test_disjoint_union_adds(ctx):
    a = graphs.rmat(9, 16, seed=11)
    b = graphs.rgg(1 << 10, seed=12)
    src = np.concatenate([np.repeat(np.arange(a.n), np.diff(a.indptr.astype(np.int64))),
                          a.n + np.repeat(np.arange(b.n), np.diff(b.indptr.astype(np.int64)))])
    dst = np.concatenate([a.indices.astype(np.int64), a.n + b.indices.astype(np.int64)])
    u = graphs.from_pairs(a.n + b.n, src, dst)
    ca, cb, cu = (graphs.cuts(x, 4, "uni") for x in (a, b, u))
    assert gpu_count(ctx, u, cu) == gpu_count(ctx, a, ca) + gpu_count(ctx, b, cb)


def test_edge_cases(ctx):
    # empty graph, one edge, one triangle
    empty = graphs.from_pairs(10, [], [])
    assert gpu_count(ctx, empty, graphs.cuts(empty, 3, "uni")) == 0
    one = csr_from_edges(2, [(0, 1)])
    assert gpu_count(ctx, one, np.array([0, 2], np.uint32)) == 0
    tri = csr_from_edges(3, [(0, 1), (1, 2), (0, 2)])
    for P in (1, 2, 3):
        assert gpu_count(ctx, tri, graphs.cuts(tri, P, "uni")) == 1
    # cut vectors with empty parts, a phantom row (cuts[P] = n + 1) and P = 64
    g = graphs.rmat(10, 16, seed=4)
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    for cuts in ([0, 0, 300, 300, 700, g.n], [0, 512, g.n + 1], list(range(0, 64 * 16, 16)) + [g.n]):
        cuts = np.array(cuts, np.uint32)
        assert oracle.count(g.n, g.indptr, g.indices, cuts) == want
        for kernel, mode in KERNEL_MODES:
            assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode) == want, (cuts[:4], kernel, mode)


def test_input_contract_errors(ctx):
    n = 4
    indptr = np.array([0, 2, 3, 3, 3], np.uint32)
    bad_rows = np.array([2, 1, 3], np.uint32)  # row 0 not increasing
    with pytest.raises(BBTcError) as e:
        Graph.upload(ctx, n, indptr, bad_rows, np.array([0, 4], np.uint32))
    assert e.value.status == -4
    dup = np.array([1, 1, 3], np.uint32)
    with pytest.raises(BBTcError):
        Graph.upload(ctx, n, indptr, dup, np.array([0, 4], np.uint32))
    big = np.array([1, 9, 3], np.uint32)
    with pytest.raises(BBTcError):
        Graph.upload(ctx, n, indptr, big, np.array([0, 4], np.uint32))
    with pytest.raises(BBTcError):  # cuts[P] < n
        Graph.upload(ctx, n, indptr, np.array([1, 2, 3], np.uint32), np.array([0, 2], np.uint32))
    with pytest.raises(BBTcError):  # decreasing cuts
        Graph.upload(ctx, n, indptr, np.array([1, 2, 3], np.uint32), np.array([0, 3, 2, 4], np.uint32))
    # the context stays usable after refused inputs
    tri = csr_from_edges(3, [(0, 1), (1, 2), (0, 2)])
    assert gpu_count(ctx, tri, np.array([0, 3], np.uint32)) == 1


def test_bbtc_driver_and_border(ctx):
    """The reference driver sequence (src/bbtc.cu:28-89) and --border values."""
    g = graphs.rmat(12, 16, seed=21)
    cuts = graphs.cuts(g, 8, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    bb = BBTc(st, st.task_list(sorted=True), st.P)
    bb.InitFlags()
    bb.SetNGPU(1)
    for border in (-1, 0, 7, len(bb.tasks), len(bb.tasks) + 5):
        bb.Separator = border
        bb.PrepareGpu()
        for _ in range(2):
            bb.ResetFlags()
            assert bb.NoOfTriangles() == want, border
    with pytest.raises(BBTcError):
        bb.SetNGPU(2)
    bb.CleanUp()


def test_task_order_does_not_matter(ctx):
    g = graphs.rmat(12, 16, seed=8)
    cuts = graphs.cuts(g, 8, "n1d")
    st = Graph.from_csr(ctx, g, cuts)
    try:
        want = oracle.count(g.n, g.indptr, g.indices, cuts)
        rng = np.random.default_rng(0)
        base = st.task_list(sorted=False)
        for _ in range(3):
            perm = base[rng.permutation(len(base))]
            assert st.count(perm) == want
        assert st.count(st.task_list(sorted=True, descending=False)) == want
    finally:
        st.free()


def test_batch_equals_alone(ctx):
    gs = [graphs.rmat(s, 8 + 4 * s % 20, seed=100 + s) for s in range(8, 14)] + [graphs.rgg(1 << 12, seed=200)]
    Ps = [4, 5, 6, 8, 12, 16, 7]
    sts = [Graph.from_csr(ctx, g, graphs.cuts(g, P, "uni")) for g, P in zip(gs, Ps)]
    try:
        alone = [st.count() for st in sts]
        for g, st, a in zip(gs, sts, alone):
            assert a == oracle.count(g.n, g.indptr, g.indices, st.cuts)
        for mode in ("persistent", "plain"):
            assert count_batch(ctx, sts, options(mode=mode)) == alone
        assert count_batch(ctx, sts[::-1]) == alone[::-1]
    finally:
        for st in sts:
            st.free()


def test_repeat_and_cuda_graph_replay(ctx):
    g = graphs.rmat(13, 16, seed=31)
    cuts = graphs.cuts(g, 8, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    try:
        for cg in (True, False):
            o = options(cuda_graph=cg)
            assert [st.count(opts=o) for _ in range(4)] == [want] * 4
            st.count_async(opts=o)
            assert st.count_wait() == want
        assert st.last_launches() == 1
        st.count(opts=options(mode="plain", cuda_graph=False))
        assert st.last_launches() > 1
    finally:
        st.free()


def test_upload_device_pointers(ctx):
    torch = pytest.importorskip("torch")
    g = graphs.rmat(12, 16, seed=41)
    cuts = graphs.cuts(g, 8, "pal")
    ip = torch.from_numpy(g.indptr.astype(np.int32)).cuda()
    ix = torch.from_numpy(g.indices.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    st = Graph.upload_device(ctx, g.n, ip.data_ptr(), ix.data_ptr(), g.m, cuts)
    try:
        assert st.count() == oracle.count(g.n, g.indptr, g.indices, cuts)
    finally:
        st.free()


def test_tile_stats_match_reference_layout(ctx):
    g = graphs.rmat(12, 16, seed=51)
    cuts = graphs.cuts(g, 8, "pal")
    st = Graph.from_csr(ctx, g, cuts)
    try:
        s = st.tile_stats()
        assert np.array_equal(s["nnz"].astype(np.uint64), oracle.tile_nnz(g.n, g.indptr, g.indices, cuts))
        assert int(s["nnz"].sum()) == g.m
        info = st.info()
        assert info.n == g.n and info.m == g.m and info.P == 8
    finally:
        st.free()


def test_device_layout_validates(ctx):
    """The device-built layout read back and checked on the host: reversed
    tiles and word rows after upload, forward tiles once built, over several
    families, partitioners, empty parts, phantom rows, P = 1 and P = 64."""
    cases = []
    g = graphs.rmat(12, 16, seed=7)
    cases += [(g, graphs.cuts(g, 8, "pal")), (g, graphs.cuts(g, 5, "n1d")), (g, graphs.cuts(g, 1, "uni")),
              (g, np.array([0, 0, 900, 900, 2500, g.n + 3], np.uint32)),
              (g, np.array(list(range(0, 64 * 64, 64)) + [g.n], np.uint32))]
    cl = graphs.chung_lu(20000, seed=3)
    cases.append((cl, graphs.cuts(cl, 16, "n1d")))
    rg = graphs.rgg(1 << 14, seed=100)
    cases.append((rg, graphs.cuts(rg, 6, "uni")))
    empty = graphs.from_pairs(10, [], [])
    cases.append((empty, graphs.cuts(empty, 3, "uni")))
    for g, cuts in cases:
        st = Graph.from_csr(ctx, g, cuts)
        try:
            st.validate()
            st.tile_stats()  # builds the forward block CSR
            st.validate()
            assert st.count() == oracle.count(g.n, g.indptr, g.indices, cuts)
        finally:
            st.free()


def test_relabelling_and_orientation_invariance(ctx):
    """Relabelled vertices (re-oriented by degree) and an orientation by id
    instead of degree count the same triangles on every kernel and mode."""
    def id_oriented(n, a, b):  # smaller id -> larger id
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        order = np.lexsort((hi, lo))
        lo, hi = lo[order], hi[order]
        indptr = np.concatenate([[0], np.cumsum(np.bincount(lo, minlength=n))]).astype(np.uint32)
        return graphs.OrientedCSR(n, indptr, hi.astype(np.uint32))

    g = graphs.rmat(12, 16, seed=13)
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    src = np.repeat(np.arange(g.n), np.diff(g.indptr.astype(np.int64)))
    dst = g.indices.astype(np.int64)
    rng = np.random.default_rng(5)
    perm = rng.permutation(g.n)
    relabelled = graphs.from_pairs(g.n, perm[src], perm[dst])
    perm = rng.permutation(g.n)
    by_id = id_oriented(g.n, perm[src], perm[dst])
    for h, part, P in ((relabelled, "pal", 7), (by_id, "uni", 5), (by_id, "n1d", 9)):
        cuts = graphs.cuts(h, P, part)
        for kernel, mode in KERNEL_MODES:
            assert gpu_count(ctx, h, cuts, kernel=kernel, mode=mode) == want, (part, kernel, mode)


def test_zero_copy_upload(ctx):
    """A host CSR in page-locked memory read by a kernel instead of the copy
    engines: used only when enabled, within the size limit and for mapped
    page-locked sources; the layout and count are the same."""
    import torch
    g = graphs.rmat(12, 16, seed=21)
    cuts = graphs.cuts(g, 6, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    ip = torch.from_numpy(g.indptr.view(np.int32)).pin_memory()
    ix = torch.from_numpy(g.indices.view(np.int32)).pin_memory()
    shifted = torch.empty(g.m + 1, dtype=torch.int32, pin_memory=True)  # a start that is not 16-byte aligned
    shifted[1:] = ix
    try:
        for limit, src, expect in ((0, ix.data_ptr(), 0), (64 << 20, ix.data_ptr(), 1), (1024, ix.data_ptr(), 0),
                                   (64 << 20, shifted.data_ptr() + 4, 1)):
            ctx.set_zero_copy(limit)
            st = Graph.upload_ptrs(ctx, g.n, ip.data_ptr(), src, g.m, cuts)
            try:
                assert st.info().zero_copy == expect, (limit, expect)
                st.validate()
                assert st.count() == want
            finally:
                st.free()
        ctx.set_zero_copy(64 << 20)
        st = Graph.from_csr(ctx, g, cuts)  # pageable numpy arrays: copied as usual
        try:
            assert st.info().zero_copy == 0
            assert st.count() == want
        finally:
            st.free()
    finally:
        ctx.set_zero_copy(0)


@pytest.mark.parametrize("bitmap_words", [16, 64, 256])
def test_mixed_pivot_kinds_in_one_queue(ctx, bitmap_words):
    """pal cuts give parts of very different widths, so one persistent launch
    runs bitmap, list and global-memory pivot tasks on the same warps; the
    shared buffer must be clean between them.  Repeated counts are identical."""
    g = graphs.rmat(15, 16, seed=13)
    cuts = graphs.cuts(g, 16, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    try:
        for unit_work in (64, 2048):
            for kernel in ("auto", "bitmap"):
                o = options(kernel=kernel, bitmap_words=bitmap_words, unit_work=unit_work, blocks_per_sm=1)
                assert [st.count(opts=o) for _ in range(3)] == [want] * 3, (kernel, bitmap_words, unit_work)
    finally:
        st.free()


@pytest.mark.parametrize("kernel", ["auto", "bitmap"])
def test_small_grids(ctx, kernel):
    """Persistent grids sized to the work: small graphs launch fewer blocks
    than the SM count."""
    for s, P in ((8, 2), (14, 8)):
        g = graphs.rmat(s, 16, seed=40 + s)
        cuts = graphs.cuts(g, P, "pal")
        want = oracle.count(g.n, g.indptr, g.indices, cuts)
        got = gpu_count(ctx, g, cuts, kernel=kernel, mode="persistent", cuda_graph=False)
        assert got == want, s


@pytest.mark.parametrize("mode", ["persistent", "plain"])
@pytest.mark.parametrize("kernel", ["bitmap", "search"])
def test_bulk_staged_pivots(ctx, kernel, mode):
    """Per-task pivot rows of 64 ids or more are staged in shared memory by a
    bulk copy (the bitmap kind sets its bitmap from the staged ids, the list
    kind searches them in place); a skewed graph cut in few parts has many
    such tile rows, at every 16-byte misalignment of their start."""
    g = graphs.rmat(16, 16, seed=1)
    for P in (2, 4, 8):
        cuts = graphs.cuts(g, P, "uni")
        # the longest row of a tile, from the host CSR: staging needs >= 64 ids
        ip, ix = g.indptr.astype(np.int64), g.indices.astype(np.int64)
        part = np.searchsorted(cuts, ix, side="right") - 1
        row = np.repeat(np.arange(g.n), np.diff(ip))
        longest = np.bincount(row * P + part).max()
        assert longest >= 64, longest
        want = oracle.count(g.n, g.indptr, g.indices, cuts)
        assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode, cuda_graph=False) == want, P


def csr_rows(n, rows):
    """A CSR from explicit sorted rows {row: [ids]} (any ids below n)."""
    idx, indptr = [], np.zeros(n + 1, np.uint32)
    for u in range(n):
        idx += list(rows.get(u, []))
        indptr[u + 1] = len(idx)
    return graphs.OrientedCSR(n, indptr, np.array(idx, np.uint32))


def random_sorted_csr(n, max_deg, seed):
    """Rows of random distinct ids below n in increasing order: ids below the
    row and self loops included (a CSR the input contract accepts that is not
    an oriented graph)."""
    rng = np.random.default_rng(seed)
    rows = [np.unique(rng.integers(0, n, size=int(d))) for d in rng.integers(0, max_deg + 1, size=n)]
    indptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32)
    return graphs.OrientedCSR(n, indptr, np.concatenate(rows).astype(np.uint32))


def test_unoriented_csr_counts_the_reference_task_sum(ctx):
    """A CSR whose rows hold ids below the row: the count is the reference's
    task sum (its tiles keep only common neighbours in column parts k >= j),
    on every kernel and mode, and equals the reference's own code."""
    cases = []
    ce = csr_rows(51, {40: [0, 50], 50: [0]})  # the reference counts 1 with P = 1
    for cuts in ([0, 51], [0, 20, 51], [0, 40, 45, 51], [0, 33, 51], [0, 41, 52]):
        cases.append((ce, np.array(cuts, np.uint32)))
    for seed, (n, deg) in enumerate([(200, 30), (1000, 60), (3000, 200)]):
        h = random_sorted_csr(n, deg, seed)
        for P, part in ((1, "uni"), (4, "uni"), (7, "n1d")):
            cases.append((h, graphs.cuts(h, P, part)))
    for g, cuts in cases:
        want = oracle.count(g.n, g.indptr, g.indices, cuts)
        if oracle.ref_available():
            assert oracle.ref_count(g.n, g.indptr, g.indices, cuts)[0] == want
        for kernel, mode in KERNEL_MODES:
            assert gpu_count(ctx, g, cuts, kernel=kernel, mode=mode) == want, (g.n, list(cuts), kernel, mode)
    assert oracle.count(ce.n, ce.indptr, ce.indices, np.array([0, 51], np.uint32)) == 1


@pytest.mark.parametrize("bitmap_words", [0, 64, 256])
def test_unoriented_wide_pivots(ctx, bitmap_words):
    """Non-oriented rows spread over a wide id range, so the fused pivots run
    as bitmap, split, list and global-memory kinds with ids below the task
    columns dropped."""
    h = random_sorted_csr(1 << 15, 120, seed=9)
    for P, part in ((3, "uni"), (8, "n1d")):
        cuts = graphs.cuts(h, P, part)
        want = oracle.count(h.n, h.indptr, h.indices, cuts)
        st = Graph.from_csr(ctx, h, cuts)
        try:
            st.validate()
            for kernel, mode in (("auto", "persistent"), ("fused", "plain"), ("bitmap", "persistent")):
                got = st.count(opts=options(kernel=kernel, mode=mode, bitmap_words=bitmap_words))
                assert got == want, (P, kernel, mode, bitmap_words)
        finally:
            st.free()


def test_batch_configuration_draw_against_oracle(ctx):
    """The batched-launch configuration's generator mix, down-scaled (512
    R-MAT graphs of scale 10-12, edge factor 8-32, and 64 random geometric
    graphs of 2^14-2^18 points, each with its own uni ncut 4-16): one
    persistent launch counts every graph as the oracle does."""
    import bench
    work = bench.batch_workload(12)
    assert len(work) == 576
    want = bench.oracle_counts(work)
    sts = [Graph.from_csr(ctx, g, c) for g, c in work]
    try:
        assert count_batch(ctx, sts) == want
    finally:
        for st in sts:
            st.free()

"""The oracle pinned before it is trusted: the C restatement equals the
reference's own CPU path (compiled from its sources into oracle/_ref), the
reference's unmodified executable, and closed-form / brute-force counts."""
import math
import os
import sys

import numpy as np
import pytest

import oracle
from bbtc_b200 import graphs

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def edges_graph(n, edges):
    return graphs.from_pairs(n, [e[0] for e in edges], [e[1] for e in edges])


@needs_ref
@pytest.mark.parametrize("scale,ef,seed", [(8, 8, 1), (10, 16, 2), (12, 16, 3), (14, 16, 4)])
@pytest.mark.parametrize("part,P", [("pal", 8), ("uni", 3), ("n1d", 16)])
def test_restatement_equals_reference(scale, ef, seed, part, P):
    g = graphs.rmat(scale, ef, seed=seed)
    cuts = graphs.cuts(g, P, part)
    ref, _ = oracle.ref_count(g.n, g.indptr, g.indices, cuts)
    assert oracle.count(g.n, g.indptr, g.indices, cuts) == ref


@needs_ref
def test_config1_against_reference_executable():
    """R-MAT scale 16, ef 16, seed 1, pal ncut 8, through the reference's own
    CLI (its reader, symmetriser, degree order, SARMA pal cuts)."""
    g = graphs.rmat(16, 16, seed=1)
    res = oracle.ref_cli(g.n, g.indptr, g.indices, "pal", 8)
    assert res["edges"] == g.m
    assert oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 8, "pal")) == res["triangles"]


@needs_ref
@pytest.mark.parametrize("part", ["uni", "n1d", "pal"])
def test_reference_executable_partitioners(part):
    g = graphs.rgg(1 << 11, seed=7)
    res = oracle.ref_cli(g.n, g.indptr, g.indices, part, 4)
    assert oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni")) == res["triangles"]


def test_brute_force_small():
    for seed in range(4):
        g = graphs.rmat(6, 6, seed=seed)
        want = oracle.brute_force(g.n, g.indptr, g.indices)
        for P in (1, 2, 5):
            assert oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, P, "uni")) == want


def test_closed_forms():
    n = 25
    kn = edges_graph(n, [(a, b) for a in range(n) for b in range(a + 1, n)])
    assert oracle.count(kn.n, kn.indptr, kn.indices, graphs.cuts(kn, 4, "uni")) == math.comb(n, 3)
    w = 30
    wheel = edges_graph(w + 1, [(0, i) for i in range(1, w + 1)] + [(i, i % w + 1) for i in range(1, w + 1)])
    assert oracle.count(wheel.n, wheel.indptr, wheel.indices, graphs.cuts(wheel, 3, "uni")) == w
    grid = edges_graph(36, [(r * 6 + c, r * 6 + c + 1) for r in range(6) for c in range(5)]
                       + [(r * 6 + c, (r + 1) * 6 + c) for r in range(5) for c in range(6)])
    assert oracle.count(grid.n, grid.indptr, grid.indices, graphs.cuts(grid, 4, "uni")) == 0


def test_partition_invariance():
    g = graphs.rmat(12, 16, seed=11)
    counts = {oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, P, part))
              for part in ("uni", "n1d", "pal") for P in (1, 2, 7, 16)}
    assert len(counts) == 1


def id_oriented(n, src, dst):
    """CSR oriented from the smaller to the larger id (not by degree)."""
    lo, hi = np.minimum(src, dst).astype(np.int64), np.maximum(src, dst).astype(np.int64)
    order = np.lexsort((hi, lo))
    lo, hi = lo[order], hi[order]
    indptr = np.concatenate([[0], np.cumsum(np.bincount(lo, minlength=n))]).astype(np.uint32)
    return graphs.OrientedCSR(n, indptr, hi.astype(np.uint32))


def test_relabelling_and_orientation_invariance():
    """Relabelled vertices (re-oriented by degree) and an orientation by id
    instead of degree give the same count: every acyclic orientation counts
    each triangle once."""
    g = graphs.rmat(11, 16, seed=13)
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    src = np.repeat(np.arange(g.n), np.diff(g.indptr.astype(np.int64)))
    dst = g.indices.astype(np.int64)
    rng = np.random.default_rng(5)
    for _ in range(2):
        perm = rng.permutation(g.n)
        h = graphs.from_pairs(g.n, perm[src], perm[dst])
        assert h.m == g.m
        assert oracle.count(h.n, h.indptr, h.indices, graphs.cuts(h, 5, "pal")) == want
    perm = rng.permutation(g.n)
    h = id_oriented(g.n, perm[src], perm[dst])
    assert h.m == g.m
    assert oracle.count(h.n, h.indptr, h.indices, graphs.cuts(h, 3, "uni")) == want


def test_plants_are_caught():
    """A planted mistake in the oracle's input changes the count (the check has teeth)."""
    g = graphs.rmat(10, 16, seed=5)
    cuts = graphs.cuts(g, 4, "uni")
    good = oracle.count(g.n, g.indptr, g.indices, cuts)
    bad = g.indices.copy()
    # drop the last entry of the longest row: removes at least one triangle edge in this graph
    d = np.diff(g.indptr.astype(np.int64))
    r = int(np.argmax(d))
    ip = g.indptr.astype(np.int64).copy()
    keep = np.ones(g.m, bool)
    keep[ip[r + 1] - 1] = False
    ip[r + 1:] -= 1
    assert oracle.count(g.n, ip.astype(np.uint32), bad[keep], cuts) != good


@pytest.mark.parametrize("scale,ef,seed", [(8, 8, 1), (12, 16, 5), (16, 16, 1), (14, 32, 9)])
def test_generator_restatement_equals_library(scale, ef, seed):
    """The oracle's own generators (oracle/graphs_oracle.c: a global key sort
    instead of the library's per-row buckets) give the library's graphs bit
    for bit, so the reference arm can build them without the library."""
    n, ip, ix = oracle.rmat(scale, ef, seed=seed)
    g = graphs.rmat(scale, ef, seed=seed)
    assert n == g.n and np.array_equal(ip, g.indptr) and np.array_equal(ix, g.indices)


@pytest.mark.parametrize("n,max_deg", [(1 << 12, 500.0), (30000, 3000.0)])
def test_chung_lu_restatement_equals_library(n, max_deg):
    _, ip, ix = oracle.chung_lu(n, seed=3, max_deg=max_deg)
    g = graphs.chung_lu(n, seed=3, max_deg=max_deg)
    assert np.array_equal(ip, g.indptr) and np.array_equal(ix, g.indices)


def random_sorted_csr(n, max_deg, seed):
    rng = np.random.default_rng(seed)
    rows = [np.unique(rng.integers(0, n, size=int(d))) for d in rng.integers(0, max_deg + 1, size=n)]
    indptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32)
    return indptr, np.concatenate(rows).astype(np.uint32)


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restatement_equals_reference_unoriented(seed):
    """CSRs the input contract accepts that are not oriented graphs (ids
    below the row, self loops): the restatement still gives the reference's
    task sum, which then is not a triangle count."""
    n = 150 * seed
    ip, ix = random_sorted_csr(n, 25, seed)
    rng = np.random.default_rng(seed)
    for P in (1, 2, 5):
        cuts = np.unique(np.concatenate([[0], rng.integers(0, n, size=P - 1), [n]])).astype(np.uint32)
        assert oracle.count(n, ip, ix, cuts) == oracle.ref_count(n, ip, ix, cuts)[0]
    rows = {40: [0, 50], 50: [0]}
    ip2 = np.zeros(52, np.uint32)
    for u in range(51):
        ip2[u + 1] = ip2[u] + len(rows.get(u, []))
    ix2 = np.array(rows[40] + rows[50], np.uint32)
    assert oracle.count(51, ip2, ix2, np.array([0, 51], np.uint32)) == 1 == \
        oracle.ref_count(51, ip2, ix2, np.array([0, 51], np.uint32))[0]


def _row_bottleneck(g, cuts):
    ip = g.indptr.astype(np.int64)
    return int(np.diff(ip[np.minimum(cuts.astype(np.int64), g.n)]).max())


@needs_ref
@pytest.mark.parametrize("make", [lambda: graphs.rmat(14, 16, seed=2), lambda: graphs.rgg(1 << 14, seed=5),
                                  lambda: graphs.chung_lu(1 << 15, seed=3, max_deg=3000.0)])
@pytest.mark.parametrize("P", [4, 8, 16])
def test_partitioners_against_sarma(make, P):
    """The library's partitioners against the reference's own (SARMA, run by
    the reference's call sequence in oracle/_ref): uni gives SARMA's cuts (the
    last is n, where SARMA puts n + 1); n1d is the optimal contiguous split of
    the row loads, so its bottleneck is at most SARMA's; pal is an
    independent probe-a-load implementation with its own sample, so its
    largest tile is compared, not its cuts (within 15 %)."""
    g = make()
    uni, ref_uni = graphs.cuts(g, P, "uni"), oracle.ref_cuts(g.n, g.indptr, g.indices, P, "uni")
    assert np.array_equal(uni[:-1], ref_uni[:-1]) and uni[-1] == g.n and ref_uni[-1] == g.n + 1
    n1d, ref_n1d = graphs.cuts(g, P, "n1d"), oracle.ref_cuts(g.n, g.indptr, g.indices, P, "n1d")
    assert _row_bottleneck(g, n1d) <= _row_bottleneck(g, ref_n1d)
    pal, ref_pal = graphs.cuts(g, P, "pal"), oracle.ref_cuts(g.n, g.indptr, g.indices, P, "pal")
    ours = int(oracle.tile_nnz(g.n, g.indptr, g.indices, pal).max())
    theirs = int(oracle.tile_nnz(g.n, g.indptr, g.indices, ref_pal).max())
    assert ours <= 1.15 * theirs, (ours, theirs)



def test_rac_equals_sarma():
    """rac (refine a cut) is deterministic: the library's cuts equal SARMA's
    (refine_a_cut::partition on the whole matrix, the reference's call
    sequence of utils.hpp:282-283, run by tests/golden/make_golden.py --rac),
    except the last cut (n here, n + 1 in the reference).  The reference's
    cuts are fixtures: its rac crashed the test process now and then (a
    segmentation fault inside SARMA's parallel loops)."""
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import RAC_CASES, RAC_P
    ref = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sarma-rac-cuts.npz"))
    for key, make in RAC_CASES.items():
        g = make()
        for P in RAC_P:
            theirs = ref[f"{key}__{P}"]
            ours = graphs.cuts(g, P, "rac")
            assert np.array_equal(ours[:-1], theirs[:-1]), (key, P, ours, theirs)
            assert ours[-1] == g.n and theirs[-1] == g.n + 1

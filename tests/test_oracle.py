"""The oracle pinned before it is trusted: the C restatement equals the
reference's own CPU path (compiled from its sources into oracle/_ref), the
reference's unmodified executable, and closed-form / brute-force counts."""
import math

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

"""Host-side input generation and cut vectors."""
import numpy as np
import pytest

from bbtc_b200 import graphs


def check_oriented(g):
    ip = g.indptr.astype(np.int64)
    assert ip[0] == 0 and ip[-1] == g.m and np.all(np.diff(ip) >= 0)
    rows = np.repeat(np.arange(g.n), np.diff(ip))
    cols = g.indices.astype(np.int64)
    assert np.all(cols > rows), "oriented low -> high"
    same = rows[1:] == rows[:-1]
    assert np.all(cols[1:][same] > cols[:-1][same]), "rows strictly increasing"
    # orientation by (degree, id): every edge points to a vertex of >= degree
    deg = np.bincount(rows, minlength=g.n) + np.bincount(cols, minlength=g.n)
    assert np.all(deg[rows] <= deg[cols])


@pytest.mark.parametrize("make", [lambda: graphs.rmat(12, 16, seed=1), lambda: graphs.rgg(1 << 12, seed=5),
                                  lambda: graphs.chung_lu(1 << 13, seed=3, max_deg=500)])
def test_generators_give_oriented_csr(make):
    a, b = make(), make()
    check_oriented(a)
    assert np.array_equal(a.indptr, b.indptr) and np.array_equal(a.indices, b.indices), "deterministic"


def test_from_pairs_cleans():
    g = graphs.from_pairs(5, [0, 1, 1, 2, 3, 3, 4], [1, 0, 1, 3, 2, 4, 4])
    # edges {0,1}, {2,3}, {3,4}; the loop (1,1), (4,4) and the reversed duplicates go
    assert g.m == 3
    check_oriented(g)


def test_rmat_size():
    g = graphs.rmat(16, 16, seed=1)
    assert g.n == 65536 and g.m_raw == 1 << 20 and 800_000 < g.m < 1_000_000


@pytest.mark.parametrize("part", ["uni", "n1d", "pal"])
@pytest.mark.parametrize("P", [1, 2, 8, 16, 33])
def test_cuts_valid(part, P):
    g = graphs.rmat(11, 16, seed=3)
    c = graphs.cuts(g, P, part).astype(np.int64)
    assert len(c) == P + 1 and c[0] == 0 and c[-1] == g.n and np.all(np.diff(c) >= 0)


def test_uniform_cuts_match_sarma_formula():
    g = graphs.rmat(10, 8, seed=1)
    assert graphs.cuts(g, 7, "uni").tolist() == [i * g.n // 7 for i in range(8)]


def test_n1d_is_balanced():
    g = graphs.rmat(14, 16, seed=2)
    P = 8
    c = graphs.cuts(g, P, "n1d").astype(np.int64)
    loads = np.diff(g.indptr.astype(np.int64)[c])
    rowmax = np.diff(g.indptr.astype(np.int64)).max()
    assert loads.max() <= max(rowmax, -(-g.m // P)) + rowmax


def test_algorithmic_bytes():
    g = graphs.from_pairs(4, [0, 0, 1], [1, 2, 2])  # one triangle, all degree 2
    d = g.out_degrees()
    rows = np.repeat(np.arange(g.n), d)
    want = 4 * g.m + 4 * int((d[rows] + d[g.indices]).sum())
    assert g.algorithmic_bytes() == want


@pytest.mark.parametrize("make", [lambda: graphs.rmat(8, 16, seed=1), lambda: graphs.rmat(13, 16, seed=2),
                                  lambda: graphs.rmat(16, 8, seed=3), lambda: graphs.rgg(1 << 13, seed=4),
                                  lambda: graphs.chung_lu(1 << 14, seed=5, max_deg=1500)])
def test_pal_sweep_probe_equals_bisection(make):
    """The sweep probe (default pal) finds the same cut positions as the
    bisection probe it replaced, for every stripe count."""
    g = make()
    for P in (1, 2, 3, 7, 16, 33, 64):
        assert np.array_equal(graphs.cuts(g, P, "pal"), graphs.cuts(g, P, "pal-bisect")), P

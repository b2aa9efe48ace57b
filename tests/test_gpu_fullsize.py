"""Full-size parity: the single-graph and skewed-degree configurations,
counted on the GPU and by the reference's own CPU path (oracle/_ref, all
host cores) on the same graph and cuts; plus size-independent properties
(every kernel and form agree, the count does not depend on the cuts)."""
import os

import pytest

import oracle
from bbtc_b200 import Graph, graphs, options

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


@pytest.fixture(scope="module")
def c2():
    g = graphs.rmat(22, 16, seed=2)
    return g, graphs.cuts(g, 16, "pal")


def test_rmat22_pal16_equals_reference(ctx, c2):
    g, cuts = c2
    st = Graph.from_csr(ctx, g, cuts)
    try:
        got = st.count()
        if oracle.ref_available():
            ref, _ = oracle.ref_count(g.n, g.indptr, g.indices, cuts, nthreads=os.cpu_count())
            assert got == ref
        else:
            assert got == oracle.count(g.n, g.indptr, g.indices, cuts)
        assert st.count(opts=options(mode="plain", cuda_graph=False)) == got
        assert st.count(opts=options(kernel="bitmap")) == got
        assert st.count(opts=options(bitmap_words=4096, warps_per_block=4)) == got
    finally:
        st.free()


def test_rmat22_other_cuts_same_count(ctx, c2):
    g, cuts = c2
    want = None
    for part, P in (("pal", 16), ("n1d", 32), ("uni", 8)):
        st = Graph.from_csr(ctx, g, graphs.cuts(g, P, part))
        c = st.count()
        st.free()
        want = c if want is None else want
        assert c == want, (part, P)


def test_chunglu8m_n1d32_equals_reference(ctx):
    g = graphs.chung_lu(1 << 23, gamma=2.1, mean_deg=20.0, max_deg=50000.0, seed=3)
    cuts = graphs.cuts(g, 32, "n1d")
    st = Graph.from_csr(ctx, g, cuts)
    try:
        got = st.count()
        if oracle.ref_available():
            ref, _ = oracle.ref_count(g.n, g.indptr, g.indices, cuts, nthreads=os.cpu_count())
            assert got == ref
        else:
            assert got == oracle.count(g.n, g.indptr, g.indices, cuts)
        assert st.count(opts=options(kernel="merge")) == got
    finally:
        st.free()

"""Host-side fault injection: any device allocation of an upload, a count, a
forward block-CSR build, a batch or a served request can be made to fail
(bbtc_debug_fail_alloc).  The call then returns BBTC_ERR_NOMEM, holds
nothing, and the library keeps working.  Nothing faults on the GPU: the
failing allocation is never made, and nothing is launched on its buffer."""
import numpy as np
import pytest

import oracle
from bbtc_b200 import BBTcError, Graph, Server, core, count_batch, graphs, options

pytestmark = pytest.mark.gpu

NOMEM = -3


@pytest.fixture(autouse=True)
def disarmed():
    core.debug_fail_alloc(-1)
    yield
    core.debug_fail_alloc(-1)


def workload(ctx, g, cuts, tasks):
    st = Graph.from_csr(ctx, g, cuts)
    try:
        whole = st.count()  # fused task rows
        st.tile_stats()  # forward block CSR
        part = st.count(tasks, opts=options(kernel="auto"))  # per-task kernels
        batch = count_batch(ctx, [st, st])
        st.validate()
        return whole, part, batch
    finally:
        st.free()


def test_every_allocation_can_fail(ctx):
    g = graphs.rmat(11, 16, seed=9)
    cuts = graphs.cuts(g, 5, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    tl = core.task_list(5)[:7].copy()
    want_part = sum(oracle.task_count(g.n, g.indptr, g.indices, cuts, int(t["ab"]), int(t["bc"]), int(t["ac"]))
                    for t in tl)
    expect = (want, want_part, [want, want])
    fired = 0
    for k in range(400):
        core.debug_fail_alloc(k)
        try:
            got = workload(ctx, g, cuts, tl)
        except BBTcError as e:
            assert e.status == NOMEM, (k, e.status, e.message)
            got = None
        left = core.debug_fail_alloc(-1)
        if left >= 0:  # the fault did not fire: every allocation passed
            assert got == expect
            break
        assert got is None, k  # the fault fired: the call failed
        fired += 1
        assert workload(ctx, g, cuts, tl) == expect, k  # and nothing is left broken
    else:
        pytest.fail("the workload made more than 400 device allocations")
    assert fired >= 10


def test_served_request_fails_alone():
    g = graphs.rmat(10, 16, seed=11)
    cuts = graphs.cuts(g, 4, "uni")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    with Server(0, loaders=1) as srv:
        warm = srv.submit_csr(g, cuts)
        assert srv.wait(warm, 60000).count == want
        srv.release(warm)
        fired = 0
        for k in range(100):
            core.debug_fail_alloc(k)
            rid = srv.submit_csr(g, cuts)
            info = srv.wait(rid, 60000)
            status, count = info.status, info.count
            srv.release(rid)
            left = core.debug_fail_alloc(-1)
            if left >= 0:
                assert status == 1 and count == want
                break
            assert status == NOMEM, (k, status)
            fired += 1
            ok = srv.submit_csr(g, cuts)
            assert srv.wait(ok, 60000).count == want, k
            srv.release(ok)
        else:
            pytest.fail("a request made more than 100 device allocations")
        assert fired >= 5
        assert srv.stats().pending == 0


@pytest.mark.parametrize("mode", ["persistent", "plain"])
@pytest.mark.parametrize("kernel", ["bitmap", "search"])
def test_staging_wait_runs_out(ctx, kernel, mode):
    """The bounded wait of the per-task kernels' shared-memory staging runs
    out (the test hook issues no copy, so the wait can only give up, with
    nothing in flight): the count returns BBTC_ERR_TIMEOUT, and the next count
    on the same context and graph is right, replayed CUDA graph included."""
    g = graphs.rmat(14, 16, seed=1)
    cuts = graphs.cuts(g, 2, "uni")  # long tile rows: many pivots of >= 64 ids are staged
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    o = options(kernel=kernel, mode=mode, cuda_graph=(mode == "persistent"))
    try:
        assert st.count(opts=o) == want
        ctx.debug_stage_timeout(4)
        try:
            with pytest.raises(BBTcError) as e:
                st.count(opts=o)
            assert e.value.status == -5, e.value.message
        finally:
            ctx.debug_stage_timeout(0)
        for _ in range(2):
            assert st.count(opts=o) == want
    finally:
        st.free()

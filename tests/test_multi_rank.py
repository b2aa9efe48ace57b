"""Multi-rank host logic on CPU: world size 2 over gloo (127.0.0.1)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from bbtc_b200 import graphs, multi


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # weak scaling: every rank counts its own graph (seed 2 + rank)
        g = graphs.rmat(11, 16, seed=2 + rank)
        cuts = graphs.cuts(g, 8, "pal")
        c = oracle.count(g.n, g.indptr, g.indices, cuts)
        m_tot, c_tot, t_max = multi.aggregate(dist, g.m, c, 0.5 + rank)
        # strong scaling: one graph, its tasks split by cost over ranks
        h = graphs.rmat(11, 16, seed=99)
        hc = graphs.cuts(h, 6, "n1d")
        P = len(hc) - 1
        tl = np.array([(i * P + j, j * P + k, i * P + k) for i in range(P) for j in range(i, P)
                       for k in range(j, P)], dtype=[("ab", np.uint32), ("bc", np.uint32), ("ac", np.uint32)])
        nnz = oracle.tile_nnz(h.n, h.indptr, h.indices, hc).astype(np.float64)
        height = np.repeat(np.diff(hc.astype(np.int64)), P).astype(np.float64)
        with np.errstate(divide="ignore", invalid="ignore"):
            deg = nnz / height
        shards = multi.shard_tasks(multi.task_costs(nnz, deg, tl), world)
        mine = sum(oracle.task_count(h.n, h.indptr, h.indices, hc, int(t["ab"]), int(t["bc"]), int(t["ac"]))
                   for t in tl[shards[rank]])
        _, shard_sum, _ = multi.aggregate(dist, 0, mine, 0.0)
        q.put((rank, g.m, c, m_tot, c_tot, t_max, shard_sum, [s.tolist() for s in shards]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    ms = [r[1] for r in res]
    cs = [r[2] for r in res]
    for r in res:
        assert r[3] == sum(ms) and r[4] == sum(cs) and r[5] == 1.5
    h = graphs.rmat(11, 16, seed=99)
    full = oracle.count(h.n, h.indptr, h.indices, graphs.cuts(h, 6, "n1d"))
    assert all(r[6] == full for r in res)
    shards = res[0][7]
    allt = sorted(t for s in shards for t in s)
    assert allt == list(range(len(allt))) and all(len(s) > 0 for s in shards)


def test_shard_tasks_balanced():
    costs = np.random.default_rng(0).pareto(1.5, size=816) + 1
    shards = multi.shard_tasks(costs, 8)
    loads = [costs[s].sum() for s in shards]
    assert sorted(np.concatenate(shards).tolist()) == list(range(816))
    assert max(loads) <= min(loads) + costs.max()

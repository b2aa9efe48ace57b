"""Hybrid GPU + CPU execution through the C ABI (bbtc_count_hybrid), against
the oracle: tasks [0, Separator) on the GPU, the rest shared with CPU workers
that take them from the tail (bb_tc.cpp:142-252).  Counts are integers:
every comparison is exact."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle
from bbtc_b200 import BBTc, BBTcError, Graph, build, graphs, options

pytestmark = pytest.mark.gpu
EXE = os.path.join(os.path.dirname(build.__file__), "bin", "bbtc")


def unoriented(n, seed):
    rng = np.random.default_rng(seed)
    rows = [np.unique(rng.integers(0, n, rng.integers(0, 12))) for _ in range(n)]
    indptr = np.zeros(n + 1, np.uint32)
    indptr[1:] = np.cumsum([len(r) for r in rows])
    return indptr, np.concatenate(rows).astype(np.uint32)


def cases():
    g = graphs.rmat(12, 16, seed=1)
    yield "rmat12-pal8", g.n, g.indptr, g.indices, graphs.cuts(g, 8, "pal")
    g = graphs.chung_lu(20000, seed=5)
    yield "chunglu-n1d6", g.n, g.indptr, g.indices, graphs.cuts(g, 6, "n1d")
    ip, ix = unoriented(500, 3)
    yield "unoriented-4", 500, ip, ix, np.array([0, 90, 91, 300, 501], np.uint32)


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: c[0])
def test_hybrid_counts_equal_oracle(ctx, case):
    name, n, ip, ix, cuts = case
    want = oracle.count(n, ip, ix, cuts)
    st = Graph.upload(ctx, n, ip, ix, cuts)
    try:
        tasks = st.task_list(sorted=True)
        nt = len(tasks)
        # each side's sum against the oracle's task sums: the GPU counts the
        # list's first gpu_tasks positions, the CPU workers the rest
        per_task = [oracle.task_count(n, ip, ix, cuts, int(t["ab"]), int(t["bc"]), int(t["ac"])) for t in tasks]
        for border in (-1, -2, 0, 7, nt + 1):
            for workers in (0, 2, 6):
                for mode in ("persistent", "plain"):
                    got, s = st.count_hybrid(ip, ix, tasks, border, workers, options(mode=mode))
                    key = (border, workers, mode)
                    assert got == want, key
                    assert s["gpu_count"] + s["cpu_count"] == want, key
                    assert s["gpu_tasks"] + s["cpu_tasks"] == nt, key
                    assert s["gpu_count"] == sum(per_task[:s["gpu_tasks"]]), key
                    assert s["cpu_count"] == sum(per_task[s["gpu_tasks"]:]), key
                    sep = nt if border in (-1, nt + 1) else nt // 2 if border == -2 else border
                    assert s["separator"] == sep and s["gpu_tasks"] >= sep, key
                    if workers == 0 or sep == nt:
                        assert s["cpu_tasks"] == 0 and s["gpu_launches"] == 1, key
        # tasks = NULL: TaskList(P) sorted heaviest first
        got, s = st.count_hybrid(ip, ix, None, 0, 3)
        assert got == want and s["gpu_tasks"] + s["cpu_tasks"] == nt
        assert st.count() == want  # the regular count is unchanged afterwards
    finally:
        st.free()


def test_cpu_workers_share_the_tail(ctx):
    """One launch per task on the GPU side and many CPU workers: both sides
    count, and the sum stays exact."""
    g = graphs.rmat(14, 16, seed=3)
    cuts = graphs.cuts(g, 16, "pal")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    try:
        tasks = st.task_list(sorted=True)
        seen_cpu = 0
        for _ in range(3):
            got, s = st.count_hybrid(g.indptr, g.indices, tasks, 0, 8, options(mode="plain"))
            assert got == want and s["gpu_tasks"] + s["cpu_tasks"] == len(tasks)
            seen_cpu += s["cpu_tasks"]
        assert seen_cpu > 0
    finally:
        st.free()


def test_hybrid_argument_and_input_errors(ctx):
    g = graphs.rmat(10, 8, seed=2)
    cuts = graphs.cuts(g, 4, "uni")
    st = Graph.from_csr(ctx, g, cuts)
    try:
        tasks = st.task_list(sorted=True)
        with pytest.raises(BBTcError) as e:
            st.count_hybrid(g.indptr, g.indices, tasks, -3, 2)
        assert e.value.status == -1
        bad = tasks.copy()
        bad[0]["ac"] = (bad[0]["ac"] + 1) % 16
        with pytest.raises(BBTcError) as e:
            st.count_hybrid(g.indptr, g.indices, bad, 0, 2)
        assert e.value.status == -1
        short = g.indptr.copy()
        short[-1] -= 1  # indptr[n] != m
        with pytest.raises(BBTcError) as e:
            st.count_hybrid(short, g.indices, tasks, 0, 2)
        assert e.value.status == -4
        unsorted = g.indices.copy()
        r = int(np.argmax(np.diff(g.indptr)))
        s0 = int(g.indptr[r])
        unsorted[s0], unsorted[s0 + 1] = unsorted[s0 + 1], unsorted[s0]
        with pytest.raises(BBTcError) as e:
            st.count_hybrid(g.indptr, unsorted, tasks, 0, 2)
        assert e.value.status == -4
        # the context and graph stay usable
        assert st.count_hybrid(g.indptr, g.indices, tasks, 0, 2)[0] == oracle.count(g.n, g.indptr, g.indices, cuts)
    finally:
        st.free()


def test_bbtc_mirror_with_cpu_workers(ctx):
    g = graphs.rmat(12, 16, seed=7)
    cuts = graphs.cuts(g, 8, "uni")
    want = oracle.count(g.n, g.indptr, g.indices, cuts)
    st = Graph.from_csr(ctx, g, cuts)
    bb = BBTc(st)
    bb.SetCpuWorkers(4, g.indptr, g.indices)
    for sep in (0, 30, -1):
        bb.Separator = sep
        assert bb.NoOfTriangles() == want
        assert bb.last_stats["gpu_tasks"] + bb.last_stats["cpu_tasks"] == len(bb.tasks)
    bb.CleanUp()


def test_cli_cpu_workers(tmp_path):
    g = graphs.rmat(12, 16, seed=4)
    path = str(tmp_path / "g.el")
    oracle.write_edge_list(path, g.n, g.indptr, g.indices)
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    # (--border -2 is refused by the reference's strict range check, utils.hpp:111-114)
    for args in (["--cpu-workers", "4", "--border", "0"], ["--cpu-workers", "-1", "--border", "30"],
                 ["--cpu-workers", "2", "--border", "-1"]):
        r = subprocess.run([EXE, "--graph", path, "--ncut", "8", "--repeat", "2", *args], capture_output=True,
                           text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        m = re.search(r"Number of Triangles:\s*(\d+)", r.stdout)
        assert m and int(m.group(1)) == want, args

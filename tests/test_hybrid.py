"""The hybrid GPU + CPU count's host side (bbtc_b200/csrc/hybrid_core.hpp) on
the CPU: the CPU workers' task count against the oracle's task sum, and the
claim protocol of bb_tc.cpp:142-252 (GPU from the head up to the first task a
CPU worker holds, CPU workers from the tail down to the Separator) with a
stand-in for the GPU side.  The GPU side itself is tested in
tests/test_gpu_with_cpu_workers.py."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from bbtc_b200 import graphs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("hy")
    exe = d / "harness"
    cxx = shutil.which("g++") or shutil.which("c++")
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-pthread", "-I", os.path.join(ROOT, "bbtc_b200", "csrc"),
                    os.path.join(ROOT, "tests", "hybrid_harness.cpp"), "-o", str(exe)], check=True)
    return exe, d


def task_list(P):
    """TaskList(P) in the reference's enumeration order (tasks.hpp:7-17)."""
    return np.array([(i * P + j, j * P + k, i * P + k) for i in range(P) for j in range(i, P) for k in range(j, P)],
                    np.uint32).reshape(-1, 3)


def write(d, name, n, indptr, indices, cuts, tasks):
    g = d / (name + ".g")
    with open(g, "wb") as f:
        np.array([n, len(cuts) - 1], np.uint32).tofile(f)
        np.array([len(indices)], np.uint64).tofile(f)
        np.asarray(indptr, np.uint32).tofile(f)
        np.asarray(indices, np.uint32).tofile(f)
        np.asarray(cuts, np.uint32).tofile(f)
    t = d / (name + ".t")
    with open(t, "wb") as f:
        np.array([len(tasks)], np.uint32).tofile(f)
        np.asarray(tasks, np.uint32).tofile(f)
    return g, t


def run(exe, *args):
    r = subprocess.run([str(exe)] + [str(a) for a in args], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (args, r.returncode, r.stdout, r.stderr)
    return r.stdout.split("\n")


def unoriented(n, seed):
    """Sorted rows that are not an orientation: ids below and above the row, self loops."""
    rng = np.random.default_rng(seed)
    rows = [np.unique(rng.integers(0, n, rng.integers(0, 12))) for _ in range(n)]
    indptr = np.zeros(n + 1, np.uint32)
    indptr[1:] = np.cumsum([len(r) for r in rows])
    return indptr, np.concatenate(rows).astype(np.uint32)


def cases():
    g = graphs.rmat(10, 16, seed=2)
    yield "rmat10-pal5", g.n, g.indptr, g.indices, graphs.cuts(g, 5, "pal")
    g = graphs.chung_lu(3000, seed=5)
    yield "chunglu-uni7", g.n, g.indptr, g.indices, graphs.cuts(g, 7, "uni")
    ip, ix = unoriented(300, 3)
    yield "unoriented-4", 300, ip, ix, np.array([0, 60, 61, 200, 301], np.uint32)  # phantom row past n
    yield "edgeless-3", 40, np.zeros(41, np.uint32), np.zeros(0, np.uint32), np.array([0, 10, 10, 40], np.uint32)
    g = graphs.rmat(8, 8, seed=3)
    yield "rmat8-one-part", g.n, g.indptr, g.indices, np.array([0, g.n + 1], np.uint32)


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: c[0])
def test_cpu_task_counts_equal_oracle(harness, case):
    exe, d = harness
    name, n, ip, ix, cuts = case
    P = len(cuts) - 1
    tasks = task_list(P)
    g, t = write(d, name, n, ip, ix, cuts, tasks)
    got = [int(x) for x in run(exe, g, t, "tasks") if x]
    want = [oracle.task_count(n, ip, ix, cuts, int(a), int(b), int(c)) for a, b, c in tasks]
    assert got == want
    assert sum(got) == oracle.count(n, ip, ix, cuts)


def sep_of(border, nt):
    if border == -1 or border > nt:
        return nt
    if border == -2:
        return nt // 2
    return border


@pytest.mark.parametrize("case", list(cases()), ids=lambda c: c[0])
def test_claim_protocol_counts_every_task_once(harness, case):
    exe, d = harness
    name, n, ip, ix, cuts = case
    P = len(cuts) - 1
    rng = np.random.default_rng(7)
    tasks = task_list(P)[rng.permutation(P * (P + 1) * (P + 2) // 6)]  # any list order
    g, t = write(d, name + "-run", n, ip, ix, cuts, tasks)
    nt = len(tasks)
    want = oracle.count(n, ip, ix, cuts)
    for border in (-1, -2, 0, 3, nt // 3, nt, nt + 5):
        for workers in (0, 1, 3, 8):
            for gpu_us in (0, 300):
                out = run(exe, g, t, "run", border, workers, gpu_us, 0)
                rc, total, gt, ct, launches, sep, gc, cc = (int(x) for x in out[0].split())
                seen = [int(x.split()[0]) for x in out[1:] if x]
                sides = "".join(x.split()[1] for x in out[1:] if x)
                key = (border, workers, gpu_us)
                # the GPU's tasks are the list's first gt positions, the CPU's the rest
                assert sides == "G" * gt + "C" * ct, key
                assert rc == 0, key
                assert total == want and gc + cc == want, key
                assert seen == [1] * nt, key
                assert sep == sep_of(border, nt), key
                assert gt + ct == nt and gt >= sep, key
                if workers == 0 or sep == nt:
                    assert ct == 0 and launches == 1, key
                if workers == 0:
                    assert gt == nt, key


def test_cpu_takes_the_tail_when_the_gpu_is_slow(harness):
    """With a slow GPU side, CPU workers count part of the shared list (the
    Separator is 1, so the GPU side launches at least once)."""
    exe, d = harness
    g0 = graphs.rmat(9, 8, seed=1)
    cuts = graphs.cuts(g0, 8, "uni")
    tasks = task_list(8)
    g, t = write(d, "slow", g0.n, g0.indptr, g0.indices, cuts, tasks)
    out = run(exe, g, t, "run", 1, 4, 5000, 0)
    rc, total, gt, ct, launches, sep, gc, cc = (int(x) for x in out[0].split())
    assert rc == 0 and total == oracle.count(g0.n, g0.indptr, g0.indices, cuts)
    assert ct > 0 and gt > 0 and launches >= 1
    assert [x for x in out[1:] if x] == ["1 G"] * gt + ["1 C"] * ct


def test_rows_breaking_the_contract_void_the_count(harness):
    """An unsorted row or an id >= n in the host CSR: the CPU workers count
    nothing and the call reports the input error."""
    exe, d = harness
    g0 = graphs.rmat(9, 8, seed=1)
    cuts = graphs.cuts(g0, 4, "uni")
    tasks = task_list(4)
    deg = np.diff(g0.indptr.astype(np.int64))
    wide = np.nonzero(deg >= 2)[0]
    # the longest row and the first and last rows with two ids: the workers'
    # row shares (split by entries) must cover every row
    for row in (int(np.argmax(deg)), int(wide[0]), int(wide[-1])):
        for kind in ("unsorted", "id"):
            ix = g0.indices.copy()
            s = int(g0.indptr[row])
            if kind == "unsorted":
                ix[s], ix[s + 1] = ix[s + 1], ix[s]
            else:
                ix[int(g0.indptr[row + 1]) - 1] = g0.n
            g, t = write(d, f"bad-{kind}-{row}", g0.n, g0.indptr, ix, cuts, tasks)
            assert run(exe, g, t, "tasks")[0] == "rows"
            for workers in (1, 3, 7):
                out = run(exe, g, t, "run", 0, workers, 0, 0)
                rc, total, gt, ct = (int(x) for x in out[0].split()[:4])
                assert rc == -4 and total == 0 and ct == 0, (kind, row, workers)


def test_gpu_failure_stops_the_workers(harness):
    """A failing GPU launch is the call's status, and nothing is summed.  The
    border keeps tasks for the GPU, so it launches at least once (with
    border 0, fast CPU workers may take every task before it starts)."""
    exe, d = harness
    g0 = graphs.rmat(9, 8, seed=1)
    cuts = graphs.cuts(g0, 6, "uni")
    tasks = task_list(6)
    g, t = write(d, "gfail", g0.n, g0.indptr, g0.indices, cuts, tasks)
    for workers in (0, 2):
        out = run(exe, g, t, "run", 5, workers, 0, 1)
        rc, total = (int(x) for x in out[0].split()[:2])
        assert rc == -2 and total == 0


def test_shape_checks(harness):
    exe, d = harness
    g0 = graphs.rmat(8, 8, seed=1)
    cuts = graphs.cuts(g0, 3, "uni")
    ip = g0.indptr.copy()
    ip[5], ip[6] = ip[6], ip[5] + 1  # row pointers not non-decreasing
    g, t = write(d, "shape", g0.n, ip, g0.indices, cuts, task_list(3))
    if not np.all(np.diff(ip.astype(np.int64)) >= 0):
        assert run(exe, g, t, "tasks")[0] == "shape"
    short = np.array(cuts, np.uint32)
    short[-1] = g0.n - 1  # cuts[P] < n
    g, t = write(d, "shape2", g0.n, g0.indptr, g0.indices, short, task_list(3))
    assert run(exe, g, t, "tasks")[0] == "shape"


def test_claim_protocol_under_thread_sanitizer(tmp_path):
    """The claim protocol's shared state (tail counter, claim flags, the CPU
    workers' start barrier, sums) has no data race: the harness built with
    ThreadSanitizer, over borders, worker counts, GPU speeds and a failing
    GPU launch, reports nothing."""
    cxx = shutil.which("g++") or shutil.which("c++")
    exe = tmp_path / "harness_tsan"
    r = subprocess.run([cxx, "-std=c++17", "-O1", "-g", "-fsanitize=thread", "-pthread", "-I",
                        os.path.join(ROOT, "bbtc_b200", "csrc"), os.path.join(ROOT, "tests", "hybrid_harness.cpp"),
                        "-o", str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.skip("no ThreadSanitizer in this compiler: " + r.stderr[-200:])
    g0 = graphs.rmat(9, 16, seed=2)
    cuts = graphs.cuts(g0, 8, "pal")
    tasks = task_list(8)[np.random.default_rng(1).permutation(120)]
    g, t = write(tmp_path, "tsan", g0.n, g0.indptr, g0.indices, cuts, tasks)
    want = oracle.count(g0.n, g0.indptr, g0.indices, cuts)
    for border in (0, 7, -2):
        for workers in (1, 6):
            for gpu_us, fail in ((0, 0), (200, 0), (0, 1)):
                b = max(border, 1) if fail and border >= 0 else border  # a GPU region: the GPU side launches
                r = subprocess.run([str(exe), str(g), str(t), "run", str(b), str(workers), str(gpu_us),
                                    str(fail)], capture_output=True, text=True, timeout=300)
                if "unexpected memory mapping" in r.stderr:
                    pytest.skip("ThreadSanitizer cannot run on this kernel's address layout")
                key = (border, workers, gpu_us, fail)
                assert r.returncode == 0 and "ThreadSanitizer" not in r.stderr, (key, r.stderr[:3000])
                rc, total = (int(x) for x in r.stdout.split()[:2])
                assert (rc, total) == ((-2, 0) if fail else (0, want)), key

"""The drop-in `bbtc` executable on a B200: same output lines as the
reference, exact counts, and the `.bbtc` cache in PIGO-CSR-v2 format."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from bbtc_b200 import build, graphs

pytestmark = pytest.mark.gpu
EXE = os.path.join(os.path.dirname(build.__file__), "bin", "bbtc")


def run(*args):
    r = subprocess.run([EXE, *args], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def field(out, name):
    m = re.search(re.escape(name) + r"\s*:?\s*(\d+)", out)
    return int(m.group(1)) if m else None


def test_edge_list_and_cache(tmp_path):
    g = graphs.rmat(12, 16, seed=4)
    path = str(tmp_path / "g.el")
    oracle.write_edge_list(path, g.n, g.indptr, g.indices)
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    out = run("--graph", path, "--ncut", "8", "--partitioner", "pal", "--border", "-1", "--repeat", "3")
    for line in ("Graph file: ", "Number of Vertices: ", "Number of Edges: ", "Number of Cuts: 8",
                 "Number of Tasks: 120", "Number of GPUs: 1", "Number of Workers: ",
                 "Partitioning and Layout construction (s) : ",
                 "Cuda Initial Memory Allocations and Stream Creation : "):
        assert line in out, line
    assert out.count("Triangle Counting Execution Time (s) : ") == 3
    assert field(out, "Number of Triangles:") == want
    assert field(out, "Number of Edges:") == g.m
    assert os.path.exists(path + ".bbtc")
    # the second run reads the cache (its text file is gone)
    os.rename(path, path + ".moved")
    open(path, "w").close()
    out2 = run("--graph", path, "--ncut", "5", "--partitioner", "n1d", "--copy-first", "--repeat", "1")
    assert field(out2, "Number of Triangles:") == want
    assert "Copy tiles to device (s) : " in out2
    out3 = run("--graph", path, "--ncut", "6", "--partitioner", "rac", "--repeat", "1")
    assert field(out3, "Number of Triangles:") == want


def test_matrix_market_one_based(tmp_path):
    g = graphs.rgg(1 << 11, seed=9)
    rows = np.repeat(np.arange(g.n), np.diff(g.indptr.astype(np.int64)))
    path = tmp_path / "g.mtx"
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate pattern symmetric\n% comment\n")
        f.write(f"{g.n} {g.n} {g.m}\n")
        for a, b in zip(rows, g.indices):
            f.write(f"{a + 1} {b + 1}\n")
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    out = run("--graph", str(path), "--ncut", "4", "--partitioner", "uni", "--repeat", "1")
    assert field(out, "Number of Triangles:") == want
    assert field(out, "Number of Vertices:") == g.n + 1  # ids stay 1-based: vertex 0 is isolated


@pytest.mark.skipif(not os.path.exists(os.path.join(oracle.HERE, "_ref", "bbtc_cpu")), reason="oracle/_ref not built")
def test_reads_the_reference_cache(tmp_path):
    """A `.bbtc` file written by the reference's own executable loads here."""
    g = graphs.rmat(11, 16, seed=6)
    path = str(tmp_path / "h.el")
    oracle.write_edge_list(path, g.n, g.indptr, g.indices)
    ref = subprocess.run([os.path.join(oracle.HERE, "_ref", "bbtc_cpu"), "--graph", path, "--ncut", "4",
                          "--repeat", "1"], capture_output=True, text=True, timeout=300)
    ref_count = field(ref.stdout, "Number of Triangles:")
    assert ref_count is not None and os.path.exists(path + ".bbtc")
    only = str(tmp_path / "only.bbtc")
    shutil.copy(path + ".bbtc", only)
    out = run("--graph", only, "--ncut", "6", "--repeat", "1")
    assert field(out, "Number of Triangles:") == ref_count

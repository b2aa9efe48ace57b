"""The host-side layout checker behind bbtc_graph_validate
(bbtc_b200/csrc/layout_check.hpp), on the CPU: a layout built on the host in
the device builder's format passes, and each planted fault is named.  The
device layouts themselves are checked in tests/test_gpu_parity.py."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from bbtc_b200 import graphs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

FAULTS = {
    "csr_unsorted": "row not strictly increasing",
    "word_mask": "empty mask",
    "word_order": "words not increasing",
    "rp_misaligned": "row segment not 16-byte aligned",
    "rp_nnz": "does not end at nnz",
    "col_misaligned": "not 16-byte aligned",
    "col_empty_segment": "empty tile has a column segment",
    "col_width": "column >= tile width",
    "col_swap": "tile row not strictly increasing",
    "col_value": "tile row differs from the source row",
    "maxdeg": "longest row differs",
    "nerows": "non-empty row count differs",
    "erow": "row index names the wrong row",
    "rec_pair": "record",
    "rec_end": "record outside the row's pairs",
    "desc_last": "pivot descriptor differs",
}


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("lc")
    exe = d / "harness"
    cxx = shutil.which("g++") or shutil.which("c++")
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "bbtc_b200", "csrc"),
                    os.path.join(ROOT, "tests", "layout_check_harness.cpp"), "-o", str(exe)], check=True)
    return exe, d


def graph_file(d, g, cuts, name):
    p = d / name
    with open(p, "wb") as f:
        np.array([g.n, len(cuts) - 1], np.uint32).tofile(f)
        np.array([g.m], np.uint64).tofile(f)
        g.indptr.astype(np.uint32).tofile(f)
        g.indices.astype(np.uint32).tofile(f)
        np.asarray(cuts, np.uint32).tofile(f)
    return p


def run(exe, path, fault):
    r = subprocess.run([str(exe), str(path), fault], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, (fault, r.returncode, r.stdout, r.stderr)
    return r.stdout.strip()


@pytest.mark.parametrize("P,part", [(1, "uni"), (4, "pal"), (7, "n1d")])
def test_clean_layout_passes(harness, P, part):
    exe, d = harness
    g = graphs.rmat(9, 8, seed=3)
    path = graph_file(d, g, graphs.cuts(g, P, part), f"g{P}.bin")
    assert run(exe, path, "none") == "OK"


def test_empty_parts_and_phantom_rows(harness):
    exe, d = harness
    g = graphs.rmat(7, 8, seed=4)
    cuts = [0, 0, 40, 40, g.n + 5]  # empty parts and rows past n
    assert run(exe, graph_file(d, g, cuts, "e.bin"), "none") == "OK"


def test_edgeless_and_id_oriented_layouts_pass(harness):
    exe, d = harness
    empty = graphs.from_pairs(10, [], [])
    assert run(exe, graph_file(d, empty, [0, 3, 7, 10], "z.bin"), "none") == "OK"
    # rows oriented by id (long rows, not degree ordered): the format does not depend on the orientation
    g = graphs.rmat(8, 16, seed=6)
    src = np.repeat(np.arange(g.n), np.diff(g.indptr.astype(np.int64)))
    lo, hi = np.minimum(src, g.indices), np.maximum(src, g.indices)
    order = np.lexsort((hi, lo))
    indptr = np.concatenate([[0], np.cumsum(np.bincount(lo[order], minlength=g.n))]).astype(np.uint32)
    h = graphs.OrientedCSR(g.n, indptr, hi[order].astype(np.uint32))
    assert run(exe, graph_file(d, h, graphs.cuts(h, 5, "uni"), "h.bin"), "none") == "OK"


@pytest.mark.parametrize("fault", sorted(FAULTS))
def test_planted_faults_are_named(harness, fault):
    exe, d = harness
    g = graphs.rmat(9, 8, seed=3)
    path = graph_file(d, g, graphs.cuts(g, 4, "pal"), "f.bin")
    out = run(exe, path, fault)
    assert out != "OK" and FAULTS[fault] in out, (fault, out)


def random_sorted_csr(n, max_deg, seed):
    """Rows of random distinct ids below n in increasing order: ids below the
    row and self loops included (not an oriented graph)."""
    rng = np.random.default_rng(seed)
    rows = [np.unique(rng.integers(0, n, size=int(d))) for d in rng.integers(0, max_deg + 1, size=n)]
    indptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32)
    return graphs.OrientedCSR(n, indptr, np.concatenate(rows).astype(np.uint32))


@pytest.mark.parametrize("P,part", [(1, "uni"), (3, "uni"), (6, "n1d")])
def test_unoriented_layout_passes(harness, P, part):
    """A CSR whose rows hold ids below the row: the reversed tiles' records
    start at the first pair that can meet the pivot's ids in the task columns."""
    exe, d = harness
    h = random_sorted_csr(300, 40, seed=P)
    assert run(exe, graph_file(d, h, graphs.cuts(h, P, part), f"u{P}.bin"), "none") == "OK"
    out = run(exe, graph_file(d, h, graphs.cuts(h, P, part), f"uf{P}.bin"), "rec_pair")
    assert out != "OK" and "record" in out

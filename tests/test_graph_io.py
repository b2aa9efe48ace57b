"""Graph files the drop-in CLI reads: edge lists, MatrixMarket and the `.bbtc`
binary CSR cache (PIGO-CSR-v2, include/utils/PIGO/pigo/impl/csr.impl.hpp:441-513
in the reference).  Malformed files are refused with -1 instead of reaching
the partitioners or the device; all of it runs on the host."""
import ctypes
import struct

import numpy as np
import pytest

from bbtc_b200 import _lib, graphs

MAGIC = b"PIGO-CSR-v2"


def lib():
    l = _lib.host()
    l.bbtcio_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_void_p)]
    l.bbtcio_write_bbtc.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_uint64]
    return l


def read(path):
    """(status, kind, indptr, indices) of one read."""
    l = lib()
    kind = ctypes.c_int(-1)
    h = ctypes.c_void_p()
    rc = l.bbtcio_read(str(path).encode(), ctypes.byref(kind), ctypes.byref(h))
    if rc != 0:
        return rc, kind.value, None, None
    n, m = ctypes.c_uint32(), ctypes.c_uint64()
    l.bbtcg_info(h, ctypes.byref(n), ctypes.byref(m), None)
    indptr = np.zeros(n.value + 1, np.uint32)
    indices = np.zeros(max(m.value, 1), np.uint32)
    l.bbtcg_copy(h, indptr.ctypes.data, indices.ctypes.data)
    l.bbtcg_free(h)
    return 0, kind.value, indptr, indices[:m.value]


def bbtc_bytes(indptr, indices, n=None, m=None, sizes=(4, 4)):
    n = len(indptr) - 1 if n is None else n
    m = len(indices) if m is None else m
    return (MAGIC + bytes(sizes) + struct.pack("<4I", n, m, n, n)
            + np.asarray(indptr, np.uint32).tobytes() + np.asarray(indices, np.uint32).tobytes())


def test_bbtc_round_trip(tmp_path):
    g = graphs.rmat(10, 8, seed=5)
    p = tmp_path / "g.el.bbtc"
    assert lib().bbtcio_write_bbtc(str(p).encode(), g.n, g.indptr.ctypes.data, g.indices.ctypes.data, g.m) == 0
    assert p.read_bytes()[:11] == MAGIC
    rc, kind, indptr, indices = read(p)
    assert rc == 0 and kind == 2
    assert np.array_equal(indptr, g.indptr) and np.array_equal(indices, g.indices)


def test_text_formats(tmp_path):
    el = tmp_path / "t.el"
    el.write_text("# comment\n0 1\n1 2 7.5\n\n2 0\n% other comment\n")
    rc, kind, indptr, indices = read(el)
    assert rc == 0 and kind == 0
    assert len(indptr) == 4 and len(indices) == 3  # one triangle, oriented
    mtx = tmp_path / "t.mtx"
    mtx.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% c\n3 3 3\n1 2\n2 3\n3 1\n")
    rc, kind, indptr, indices = read(mtx)
    assert rc == 0 and kind == 1
    assert len(indptr) == 5 and len(indices) == 3  # 1-based ids kept: vertex 0 is isolated


@pytest.mark.parametrize("case", ["truncated", "label8", "indptr0", "decreasing", "end_ne_m", "id_ge_n",
                                  "unsorted", "duplicate", "short_header"])
def test_malformed_bbtc_is_refused(tmp_path, case):
    indptr = [0, 2, 3, 3]
    indices = [1, 2, 2]
    good = bbtc_bytes(indptr, indices)
    data = {
        "truncated": good[:-4],
        "label8": bbtc_bytes(indptr, indices, sizes=(8, 8)),
        "indptr0": bbtc_bytes([1, 2, 3, 3], indices),
        "decreasing": bbtc_bytes([0, 2, 1, 3], indices),
        "end_ne_m": bbtc_bytes([0, 2, 3, 2], indices[:3]),
        "id_ge_n": bbtc_bytes(indptr, [1, 3, 2]),
        "unsorted": bbtc_bytes(indptr, [2, 1, 2]),
        "duplicate": bbtc_bytes(indptr, [1, 1, 2]),
        "short_header": good[:20],
    }[case]
    p = tmp_path / "bad.bbtc"
    p.write_bytes(data)
    assert read(p)[0] == -1
    p.write_bytes(good)
    assert read(p)[0] == 0


@pytest.mark.parametrize("text,name", [("0 1\nx 2\n", "t.el"), ("0\n", "t.el"), ("0 99999999999\n", "t.el"),
                                       ("%%MatrixMarket matrix array real general\n2 2\n", "t.mtx"),
                                       ("%%MatrixMarket matrix coordinate pattern general\n% c\nfoo\n", "t.mtx")])
def test_malformed_text_is_refused(tmp_path, text, name):
    p = tmp_path / name
    p.write_text(text)
    assert read(p)[0] == -1


def test_missing_file(tmp_path):
    assert read(tmp_path / "none.el")[0] == -1


def test_text_reader_agrees_with_the_reference_reader(tmp_path):
    """A messy edge list (random directions, pairs given both ways, self loops,
    comments, weight columns) read by this reader and by the reference's
    unmodified executable: the same edge count and triangle count.  (Lines
    repeated verbatim are left out: the reference keeps them as parallel
    edges, PIGO pigo/impl/csr.impl.hpp:51, this reader drops them.)"""
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(3)
    g = graphs.rmat(10, 8, seed=9)
    src = np.repeat(np.arange(g.n), np.diff(g.indptr.astype(np.int64)))
    lines = []
    for u, v in zip(src.tolist(), g.indices.tolist()):
        if rng.random() < 0.5:
            u, v = v, u
        lines.append(f"{u} {v}" + (f" {int(rng.integers(1, 9))}" if rng.random() < 0.3 else ""))
        if rng.random() < 0.2:
            lines.append(f"{v} {u}")
    lines += [f"{s} {s}" for s in rng.integers(0, g.n, 20).tolist()]
    rng.shuffle(lines)
    text = "# comment\n% another comment\n" + "\n".join(lines) + "\n"
    p = tmp_path / "messy.el"
    p.write_text(text)
    rc, kind, indptr, indices = read(p)
    assert rc == 0 and kind == 0 and len(indices) == g.m
    n = len(indptr) - 1
    cuts = graphs.cuts(graphs.OrientedCSR(n, indptr, indices), 4, "pal")
    ours = oracle.count(n, indptr, indices, cuts)
    ref = oracle.ref_cli(0, None, None, "pal", 4, text=text)
    assert ref["edges"] == len(indices)
    assert ref["triangles"] == ours == oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "pal"))


def test_matrix_market_agrees_with_the_reference_reader(tmp_path):
    """A MatrixMarket coordinate file (1-based ids kept, so vertex 0 is
    isolated; a value column) read by both readers."""
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    g = graphs.rmat(9, 16, seed=4)
    src = np.repeat(np.arange(g.n), np.diff(g.indptr.astype(np.int64)))
    body = "\n".join(f"{v + 1} {u + 1} 1.0" for u, v in zip(src.tolist(), g.indices.tolist()))
    text = (f"%%MatrixMarket matrix coordinate real symmetric\n% comment\n{g.n} {g.n} {g.m}\n" + body + "\n")
    p = tmp_path / "g.mtx"
    p.write_text(text)
    rc, kind, indptr, indices = read(p)
    assert rc == 0 and kind == 1 and len(indices) == g.m
    n = len(indptr) - 1
    ours = oracle.count(n, indptr, indices, graphs.cuts(graphs.OrientedCSR(n, indptr, indices), 4, "uni"))
    ref = oracle.ref_cli(0, None, None, "uni", 4, text=text, suffix=".mtx")
    assert ref["edges"] == len(indices) and ref["triangles"] == ours


def test_bbtc_caches_cross_load_with_the_reference(tmp_path):
    """A `.bbtc` cache the reference's executable writes loads here (its valid
    oriented CSR passes the reader's contract check), and one written here
    loads in the reference's executable: same edges and triangles both ways."""
    import os
    import shutil
    import subprocess
    import oracle
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built")
    exe = os.path.join(oracle.HERE, "_ref", "bbtc_cpu")
    g = graphs.rmat(11, 16, seed=6)
    want = oracle.count(g.n, g.indptr, g.indices, graphs.cuts(g, 4, "uni"))
    # reference -> here
    path = str(tmp_path / "h.el")
    oracle.write_edge_list(path, g.n, g.indptr, g.indices)
    subprocess.run([exe, "--graph", path, "--ncut", "4", "--repeat", "1"], capture_output=True, text=True,
                   timeout=300, check=True)
    theirs = tmp_path / "theirs.bbtc"
    shutil.copy(path + ".bbtc", theirs)
    rc, kind, indptr, indices = read(theirs)
    assert rc == 0 and kind == 2 and len(indices) == g.m
    n = len(indptr) - 1
    assert oracle.count(n, indptr, indices, graphs.cuts(graphs.OrientedCSR(n, indptr, indices), 3, "uni")) == want
    # here -> reference
    ours = tmp_path / "ours.bbtc"
    assert lib().bbtcio_write_bbtc(str(ours).encode(), g.n, g.indptr.ctypes.data, g.indices.ctypes.data, g.m) == 0
    out = subprocess.run([exe, "--graph", str(ours), "--ncut", "5", "--repeat", "1"], capture_output=True,
                         text=True, timeout=300, check=True).stdout
    import re
    assert int(re.search(r"Number of Triangles: (\d+)", out).group(1)) == want
    assert int(re.search(r"Number of Edges: (\d+)", out).group(1)) == g.m

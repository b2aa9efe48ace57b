"""Parity checkers for the counting path.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this package, and only as the checker / the timed reference CPU path.  The
library (bbtc_b200) never imports it.

* :func:`count` -- the C restatement of the reference's CPU path
  (oracle/tc_oracle.c, built to oracle/lib/liboracle.so).
* :func:`ref_count` -- the reference's own CPU path compiled from its sources
  (oracle/ref_harness.cpp -> oracle/_ref/libbbtc_ref.so).
* :func:`ref_cli` -- the reference's unmodified CPU executable
  (oracle/_ref/bbtc_cpu) on an edge-list file.
* :func:`ref_cuts` -- the reference's own SARMA cut vector (oracle/_ref).
* :func:`rmat`, :func:`chung_lu` -- the benchmark graphs from a restatement of
  the library's generators (oracle/graphs_oracle.c), so the timed reference
  path loads none of the library's code.
* :func:`brute_force` -- pure-Python count over all vertex triples, tiny graphs.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
import tempfile
from itertools import combinations

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_libs: dict[str, ctypes.CDLL] = {}


def reference_dir() -> str | None:
    """The reference's source tree: $BBTC_REFERENCE, else the checkout beside
    this repository (``../reference``) when it holds the reference's sources."""
    for d in (os.environ.get("BBTC_REFERENCE"), os.path.join(os.path.dirname(HERE), "..", "reference")):
        if d and os.path.exists(os.path.join(d, "src", "bbtc.cpp")):
            return os.path.realpath(d)
    return None


def build() -> None:
    """Compile the restatement and, when the reference tree is present, oracle/_ref."""
    ref = reference_dir()
    subprocess.run(["make", "-s", "-C", HERE] + ([f"REF={ref}"] if ref else []), check=True)


def _load(rel: str) -> ctypes.CDLL:
    if rel not in _libs:
        path = os.path.join(HERE, rel)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing; run `make -C oracle`")
        _libs[rel] = ctypes.CDLL(path)
    return _libs[rel]


def _p(a: np.ndarray) -> ctypes.c_void_p:
    return a.ctypes.data_as(ctypes.c_void_p)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def count(n: int, indptr, indices, cuts, nthreads: int = 0) -> int:
    """Reference CPU path, restated (tc_oracle.c: oracle_count)."""
    lib = _load("lib/liboracle.so")
    indptr, indices, cuts = _u32(indptr), _u32(indices), _u32(cuts)
    out = ctypes.c_uint64()
    lib.oracle_count.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                 ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
    rc = lib.oracle_count(n, _p(indptr), _p(indices), _p(cuts), len(cuts) - 1, nthreads, ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(f"oracle_count failed ({rc})")
    return out.value


def task_count(n: int, indptr, indices, cuts, ab: int, bc: int, ac: int) -> int:
    """One task's sum over the reference layout (sparse-task merge)."""
    lib = _load("lib/liboracle.so")
    indptr, indices, cuts = _u32(indptr), _u32(indices), _u32(cuts)
    out = ctypes.c_uint64()
    lib.oracle_task_count.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.POINTER(ctypes.c_uint64)]
    rc = lib.oracle_task_count(n, _p(indptr), _p(indices), _p(cuts), len(cuts) - 1, ab, bc, ac, ctypes.byref(out))
    if rc != 0:
        raise RuntimeError(f"oracle_task_count failed ({rc})")
    return out.value


def tile_nnz(n: int, indptr, indices, cuts) -> np.ndarray:
    lib = _load("lib/liboracle.so")
    indptr, indices, cuts = _u32(indptr), _u32(indices), _u32(cuts)
    P = len(cuts) - 1
    out = np.zeros(P * P, dtype=np.uint64)
    lib.oracle_tile_nnz.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_uint32, ctypes.c_void_p]
    rc = lib.oracle_tile_nnz(n, _p(indptr), _p(indices), _p(cuts), P, _p(out))
    if rc != 0:
        raise RuntimeError(f"oracle_tile_nnz failed ({rc})")
    return out


def _take_csr(lib, n: int, m: int, ip, ix) -> tuple[int, np.ndarray, np.ndarray]:
    try:
        indptr = np.ctypeslib.as_array(ctypes.cast(ip, ctypes.POINTER(ctypes.c_uint32)), (n + 1,)).copy()
        indices = (np.ctypeslib.as_array(ctypes.cast(ix, ctypes.POINTER(ctypes.c_uint32)), (m,)).copy()
                   if m else np.zeros(0, np.uint32))
    finally:
        lib.oracle_free(ip)
        lib.oracle_free(ix)
    return n, indptr, indices


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1) -> tuple[int, np.ndarray, np.ndarray]:
    """R-MAT graph, cleaned and oriented (graphs_oracle.c: oracle_rmat): the
    same graph as bbtc_b200.graphs.rmat, built by independent code.  Returns
    (n, indptr, indices)."""
    lib = _load("lib/liboracle.so")
    lib.oracle_rmat.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint64),
                                ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]
    lib.oracle_free.argtypes = [ctypes.c_void_p]
    n, m = ctypes.c_uint32(), ctypes.c_uint64()
    ip, ix = ctypes.c_void_p(), ctypes.c_void_p()
    rc = lib.oracle_rmat(scale, edge_factor, a, b, c, seed, ctypes.byref(n), ctypes.byref(m), ctypes.byref(ip),
                         ctypes.byref(ix))
    if rc != 0:
        raise RuntimeError(f"oracle_rmat failed ({rc})")
    return _take_csr(lib, n.value, m.value, ip, ix)


def chung_lu(n: int, gamma: float = 2.1, mean_deg: float = 20.0, max_deg: float = 50000.0,
             seed: int = 3) -> tuple[int, np.ndarray, np.ndarray]:
    """Chung-Lu graph, cleaned and oriented (graphs_oracle.c: oracle_chung_lu):
    the same graph as bbtc_b200.graphs.chung_lu.  Returns (n, indptr, indices)."""
    lib = _load("lib/liboracle.so")
    lib.oracle_chung_lu.argtypes = [ctypes.c_uint32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                    ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_void_p)]
    lib.oracle_free.argtypes = [ctypes.c_void_p]
    m = ctypes.c_uint64()
    ip, ix = ctypes.c_void_p(), ctypes.c_void_p()
    rc = lib.oracle_chung_lu(n, gamma, mean_deg, max_deg, seed, ctypes.byref(m), ctypes.byref(ip), ctypes.byref(ix))
    if rc != 0:
        raise RuntimeError(f"oracle_chung_lu failed ({rc})")
    return _take_csr(lib, n, m.value, ip, ix)


PARTITIONERS = {"uni": 0, "n1d": 1, "pal": 2, "rac": 3}


def ref_cuts(n: int, indptr, indices, ncut: int, partitioner: str = "pal") -> np.ndarray:
    """The reference's own cut vector (oracle/_ref/libbbtc_ref.so: ref_cuts),
    computed by its SARMA call sequence; cuts[ncut] = n + 1 as the reference sets it."""
    lib = _load("_ref/libbbtc_ref.so")
    indptr, indices = _u32(indptr), _u32(indices)
    out = np.zeros(ncut + 1, dtype=np.uint32)
    lib.ref_cuts.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int,
                             ctypes.c_void_p]
    rc = lib.ref_cuts(n, _p(indptr), _p(indices), ncut, PARTITIONERS[partitioner], _p(out))
    if rc != 0:
        raise RuntimeError(f"ref_cuts failed ({rc})")
    return out


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libbbtc_ref.so"))


def ref_count(n: int, indptr, indices, cuts, nthreads: int = 0, repeat: int = 1) -> tuple[int, list[float]]:
    """The reference's own CPU path (oracle/_ref/libbbtc_ref.so); returns the
    count and the per-repeat NoOfTriangles() wall times in seconds."""
    lib = _load("_ref/libbbtc_ref.so")
    indptr, indices, cuts = _u32(indptr), _u32(indices), _u32(cuts)
    out = ctypes.c_uint64()
    secs = np.zeros(repeat, dtype=np.float64)
    lib.ref_count.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                              ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p]
    rc = lib.ref_count(n, _p(indptr), _p(indices), _p(cuts), len(cuts) - 1, nthreads, repeat, ctypes.byref(out),
                       _p(secs))
    if rc != 0:
        raise RuntimeError(f"ref_count failed ({rc})")
    return out.value, secs.tolist()


def write_edge_list(path: str, n: int, indptr, indices) -> None:
    """One line `u v` per undirected edge (each edge once: the reference's
    reader does not drop repeated lines)."""
    indptr = np.asarray(indptr, dtype=np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(indptr))
    np.savetxt(path, np.stack([rows, np.asarray(indices, dtype=np.int64)], axis=1), fmt="%d")


def ref_cli(n: int, indptr, indices, partitioner: str = "pal", ncut: int = 8, nthreads: int = 0,
            extra: tuple[str, ...] = (), text: str | None = None, suffix: str = ".el") -> dict:
    """Run the reference's unmodified CPU executable on the graph written as an
    edge list (or on `text`, a graph file's contents, read by the reference's
    own reader); returns the parsed output fields.  The border stays at the CPU
    build's default 0: `--border -1` sets Separator = |T| (src/bbtc.cpp:139-141),
    which leaves no task for the CPU workers (bb_tc.cpp:187-196) and prints 0."""
    exe = os.path.join(HERE, "_ref", "bbtc_cpu")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g" + suffix)
        if text is None:
            write_edge_list(path, n, indptr, indices)
        else:
            with open(path, "w") as f:
                f.write(text)
        env = dict(os.environ)
        if nthreads > 0:
            env["OMP_NUM_THREADS"] = str(nthreads)
        res = subprocess.run([exe, "--graph", path, "--partitioner", partitioner, "--ncut", str(ncut),
                              "--repeat", "1", *extra],
                             capture_output=True, text=True, env=env, timeout=600)
    out = res.stdout
    m = re.search(r"Number of Triangles: (\d+)", out)
    if not m:
        raise RuntimeError(f"reference CLI failed:\n{out}\n{res.stderr}")
    fields = {"triangles": int(m.group(1)), "stdout": out}
    me = re.search(r"Number of Edges: (\d+)", out)
    if me:
        fields["edges"] = int(me.group(1))
    return fields


def write_bbtc(path: str, n: int, indptr, indices) -> None:
    """The oriented CSR as a PIGO-CSR-v2 `.bbtc` file, the reference's cache
    format (include/utils/utils.hpp:260-268), which it loads as the oriented
    graph without re-reading text."""
    indptr = np.ascontiguousarray(indptr, dtype=np.uint32)
    indices = np.ascontiguousarray(indices, dtype=np.uint32)
    with open(path, "wb") as f:
        f.write(b"PIGO-CSR-v2")
        f.write(bytes([4, 4]))
        f.write(np.array([n, len(indices), n, n], dtype=np.uint32).tobytes())
        f.write(indptr.tobytes())
        f.write(indices.tobytes())


def ref_gpu_cli(n: int, indptr, indices, partitioner: str = "pal", ncut: int = 16, repeat: int = 5,
                timeout: int = 900) -> dict:
    """The reference's unmodified CUDA executable (oracle/_ref/bbtc_gpu):
    `--ngpu 1 --border -1 --copy-first`, its one-launch-per-task GPU form.
    Returns the count and its "Triangle Counting Execution Time (s)" lines."""
    exe = os.path.join(HERE, "_ref", "bbtc_gpu")
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "g.bbtc")
        write_bbtc(path, n, indptr, indices)
        res = subprocess.run([exe, "--graph", path, "--partitioner", partitioner, "--ncut", str(ncut), "--ngpu", "1",
                              "--border", "-1", "--copy-first", "--repeat", str(repeat)],
                             capture_output=True, text=True, timeout=timeout)
    out = res.stdout
    m = re.search(r"Number of Triangles: (\d+)", out)
    if not m:
        raise RuntimeError(f"reference GPU executable failed:\n{out}\n{res.stderr}")
    times = [float(x) for x in re.findall(r"Triangle Counting Execution Time \(s\) : ([0-9.]+)", out)]
    copy = [float(x) for x in re.findall(r"Copy tiles to device \(s\) : ([0-9.]+)", out)]
    layout = re.search(r"Partitioning and Layout construction \(s\) : ([0-9.]+)", out)
    return {"triangles": int(m.group(1)), "count_seconds": times, "copy_seconds": copy,
            "layout_seconds": float(layout.group(1)) if layout else None, "stdout": out}


def brute_force(n: int, indptr, indices) -> int:
    """Triangles of the undirected graph the CSR represents, by checking every
    vertex triple (tiny graphs only)."""
    adj = [set() for _ in range(n)]
    indptr = np.asarray(indptr)
    indices = np.asarray(indices)
    for u in range(n):
        for v in indices[indptr[u]:indptr[u + 1]]:
            v = int(v)
            if v != u:
                adj[u].add(v)
                adj[v].add(u)
    t = 0
    for a, b, c in combinations(range(n), 3):
        if b in adj[a] and c in adj[a] and c in adj[b]:
            t += 1
    return t

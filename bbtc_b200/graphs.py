"""Seeded synthetic graphs in the counting path's input form.

Every generator returns an :class:`OrientedCSR`: symmetrised, without
self-loops or duplicate edges, relabelled by ascending (degree, id) and
oriented from the lower to the higher id, rows sorted -- the graph the
reference builds before partitioning (include/utils/utils.hpp:172-258 and
SARMA csr_matrix.hpp:503-584).  The work is done by ``libbbtc_host.so``
(bbtc_b200/csrc/graphgen.cpp).
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class OrientedCSR:
    n: int
    indptr: np.ndarray  # uint32[n+1]
    indices: np.ndarray  # uint32[m]
    m_raw: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def m(self) -> int:
        return int(self.indices.shape[0])

    def out_degrees(self) -> np.ndarray:
        return np.diff(self.indptr.astype(np.int64))

    def algorithmic_bytes(self) -> int:
        """B_alg = 4 m + 4 * sum over oriented edges (u, v) of (d+(u) + d+(v)).

        The bytes a merge intersection streams: one column word per edge plus
        both out-lists per edge.  It does not depend on the cuts or kernel."""
        d = self.out_degrees()
        rows = np.repeat(np.arange(self.n, dtype=np.int64), d)
        s = int(d[rows].sum()) + int(d[self.indices.astype(np.int64)].sum())
        return 4 * self.m + 4 * s

    def fused_bytes(self, cuts) -> dict:
        """Bytes one count by fused task rows reads at least, each byte once
        per use (no reuse through the caches), for a CSR oriented from lower
        to higher ids:

        * 8 per streamed (32-id word, bit mask) pair: in-edge (u, v) streams
          the pairs of N+(u) from the one holding v to the row's end;
        * 8 per in-edge record (first pair, end pair);
        * per pivot visit -- vertex v once per row part i that holds one of
          its in-neighbours (reversed tile (part(v), i)) -- its word pairs
          (8 each) and 28 bytes of row pointers and first / last ids.

        Returns the total and its parts."""
        n, m = self.n, self.m
        ip = self.indptr.astype(np.int64)
        ix = self.indices
        if m == 0:
            return {"bytes": 0, "pairs_streamed": 0, "pivot_visits": 0, "pivot_pairs": 0, "records": 0}
        w = ix >> 5
        flags = np.empty(m, dtype=np.int64)
        flags[0] = 1
        flags[1:] = w[1:] != w[:-1]
        starts = ip[:-1][ip[:-1] < ip[1:]]
        flags[starts] = 1  # a row's first id opens a pair
        cf = np.zeros(m + 1, dtype=np.int64)
        np.cumsum(flags, out=cf[1:])
        del flags
        wptr = cf[ip]  # pairs before each row
        deg = np.diff(ip)
        # sum over edges e of (end pair of its row - pair holding e) = sum_u d(u) wptr[u+1] - sum_e (cf[e+1] - 1)
        streamed = int((deg * wptr[1:]).sum()) - int(cf[1:].sum()) + m
        del cf
        cuts = np.asarray(cuts, dtype=np.int64)
        P = len(cuts) - 1
        part_of_row = np.searchsorted(cuts, np.arange(n, dtype=np.int64), side="right") - 1
        seen = np.zeros((n, P), dtype=np.uint8)
        src_part = np.repeat(part_of_row, deg)
        seen[ix.astype(np.int64), src_part] = 1
        del src_part
        visits_per_v = seen.sum(axis=1, dtype=np.int64)
        del seen
        wn = np.diff(wptr)
        visits = int(visits_per_v.sum())
        pivot_pairs = int((visits_per_v * wn).sum())
        total = 8 * streamed + 8 * m + 8 * pivot_pairs + 28 * visits
        return {"bytes": total, "pairs_streamed": streamed, "pivot_visits": visits, "pivot_pairs": pivot_pairs,
                "records": m}


def _take(handle: ctypes.c_void_p, name: str, meta: dict) -> OrientedCSR:
    lib = _lib.host()
    n = ctypes.c_uint32()
    m = ctypes.c_uint64()
    m_raw = ctypes.c_uint64()
    try:
        _lib.check_gen(lib.bbtcg_info(handle, ctypes.byref(n), ctypes.byref(m), ctypes.byref(m_raw)))
        indptr = np.empty(n.value + 1, dtype=np.uint32)
        indices = np.empty(m.value, dtype=np.uint32)
        _lib.check_gen(lib.bbtcg_copy(handle, indptr.ctypes.data_as(ctypes.c_void_p),
                                      indices.ctypes.data_as(ctypes.c_void_p)))
    finally:
        lib.bbtcg_free(handle)
    return OrientedCSR(n.value, indptr, indices, m_raw.value, name, meta)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1) -> OrientedCSR:
    """R-MAT with `edge_factor << scale` pairs over 2**scale ids."""
    lib = _lib.host()
    h = ctypes.c_void_p()
    _lib.check_gen(lib.bbtcg_rmat(int(scale), int(edge_factor), float(a), float(b), float(c),
                                  ctypes.c_uint64(seed), ctypes.byref(h)))
    return _take(h, f"rmat-s{scale}-ef{edge_factor}-seed{seed}",
                 dict(kind="rmat", scale=scale, edge_factor=edge_factor, a=a, b=b, c=c, seed=seed))


def chung_lu(n: int, gamma: float = 2.1, mean_deg: float = 20.0, max_deg: float = 50000.0,
             seed: int = 3) -> OrientedCSR:
    """Chung-Lu expected-degree graph with a power-law weight sequence."""
    lib = _lib.host()
    h = ctypes.c_void_p()
    _lib.check_gen(lib.bbtcg_chung_lu(ctypes.c_uint32(n), float(gamma), float(mean_deg),
                                      float(max_deg), ctypes.c_uint64(seed), ctypes.byref(h)))
    return _take(h, f"chunglu-n{n}-g{gamma}-seed{seed}",
                 dict(kind="chung_lu", n=n, gamma=gamma, mean_deg=mean_deg, max_deg=max_deg, seed=seed))


def rgg(n: int, radius: float | None = None, mean_deg: float = 12.0, seed: int = 100) -> OrientedCSR:
    """Random geometric graph in the unit square; radius defaults to the one
    giving expected mean degree `mean_deg` (r = sqrt(mean_deg / (pi n)))."""
    if radius is None:
        radius = math.sqrt(mean_deg / (math.pi * n))
    lib = _lib.host()
    h = ctypes.c_void_p()
    _lib.check_gen(lib.bbtcg_rgg(ctypes.c_uint32(n), float(radius), ctypes.c_uint64(seed), ctypes.byref(h)))
    return _take(h, f"rgg-n{n}-seed{seed}", dict(kind="rgg", n=n, radius=radius, seed=seed))


def from_pairs(n: int, src, dst, name: str = "pairs") -> OrientedCSR:
    """Clean and orient an arbitrary list of pairs (ids < n)."""
    lib = _lib.host()
    s = np.ascontiguousarray(src, dtype=np.uint32)
    d = np.ascontiguousarray(dst, dtype=np.uint32)
    if s.shape != d.shape:
        raise ValueError("src and dst differ in length")
    h = ctypes.c_void_p()
    _lib.check_gen(lib.bbtcg_from_pairs(ctypes.c_uint32(n), s.ctypes.data_as(ctypes.c_void_p),
                                        d.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint64(s.size),
                                        ctypes.byref(h)))
    return _take(h, name, dict(kind="pairs"))


PARTITIONERS = {"uni": 0, "n1d": 1, "pal": 2, "pal-bisect": 3, "rac": 4}  # pal-bisect: same cuts as pal, slower probe
PAL_SEED = 1091467301  # the sampling seed the reference passes (include/utils/utils.hpp:272)


def cuts(g: OrientedCSR, ncut: int, partitioner: str = "pal", seed: int = PAL_SEED) -> np.ndarray:
    """Symmetric cut vector (ncut+1 entries, cuts[0]=0, cuts[-1]=n) from the
    uni / n1d / pal / rac partitioners (bbtc_b200/csrc/partition.cpp)."""
    if partitioner not in PARTITIONERS:
        raise ValueError(f"unknown partitioner {partitioner!r}; expected one of {sorted(PARTITIONERS)}")
    if ncut < 1:
        raise ValueError("ncut must be >= 1")
    lib = _lib.host()
    out = np.empty(ncut + 1, dtype=np.uint32)
    _lib.check_gen(lib.bbtcp_cuts(PARTITIONERS[partitioner], ctypes.c_uint32(g.n),
                                  g.indptr.ctypes.data_as(ctypes.c_void_p),
                                  g.indices.ctypes.data_as(ctypes.c_void_p), ctypes.c_uint32(ncut),
                                  ctypes.c_uint64(seed), out.ctypes.data_as(ctypes.c_void_p)))
    return out

"""Loaders for the in-tree shared libraries (built by ``bbtc_b200/build.py``).

A missing library is an error: there is no fallback path.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "lib")

_lock = threading.Lock()
_cache: dict[str, ctypes.CDLL] = {}


class BuildMissing(RuntimeError):
    pass


def _load(name: str) -> ctypes.CDLL:
    with _lock:
        if name in _cache:
            return _cache[name]
        path = os.path.join(LIBDIR, name)
        if not os.path.exists(path):
            raise BuildMissing(f"{path} is not built; run `python -m bbtc_b200.build` first")
        lib = ctypes.CDLL(path)
        _cache[name] = lib
        return lib


def host() -> ctypes.CDLL:
    """Host library: graph generators and cut-vector partitioners."""
    lib = _load("libbbtc_host.so")
    if not getattr(lib, "_typed", False):
        c = ctypes
        lib.bbtcg_rmat.argtypes = [c.c_int, c.c_int, c.c_double, c.c_double, c.c_double, c.c_uint64,
                                   c.POINTER(c.c_void_p)]
        lib.bbtcg_chung_lu.argtypes = [c.c_uint32, c.c_double, c.c_double, c.c_double, c.c_uint64,
                                       c.POINTER(c.c_void_p)]
        lib.bbtcg_rgg.argtypes = [c.c_uint32, c.c_double, c.c_uint64, c.POINTER(c.c_void_p)]
        lib.bbtcg_from_pairs.argtypes = [c.c_uint32, c.c_void_p, c.c_void_p, c.c_uint64,
                                         c.POINTER(c.c_void_p)]
        lib.bbtcg_info.argtypes = [c.c_void_p, c.POINTER(c.c_uint32), c.POINTER(c.c_uint64),
                                   c.POINTER(c.c_uint64)]
        lib.bbtcg_copy.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p]
        lib.bbtcg_free.argtypes = [c.c_void_p]
        lib.bbtcp_cuts.argtypes = [c.c_int, c.c_uint32, c.c_void_p, c.c_void_p, c.c_uint32, c.c_uint64,
                                   c.c_void_p]
        for f in ("bbtcp_cuts", "bbtcg_rmat", "bbtcg_chung_lu", "bbtcg_rgg", "bbtcg_from_pairs", "bbtcg_info",
                  "bbtcg_copy", "bbtcg_free"):
            getattr(lib, f).restype = c.c_int
        lib._typed = True
    return lib


_GEN_ERRORS = {-1: "bad argument", -2: "out of host memory", -3: "graph has 2^32 or more edges"}


def check_gen(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"graph generator failed: {_GEN_ERRORS.get(rc, rc)}")

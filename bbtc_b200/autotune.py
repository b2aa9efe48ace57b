"""Autotuner front end: the sweep runs in the library (bbtc_autotune), the
winners are kept in a small JSON cache keyed by GPU name and graph statistics.

Cache file: $BBTC_AUTOTUNE_CACHE, else ~/.cache/bbtc_b200/autotune.json.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import threading

import numpy as np

from . import core

_lock = threading.Lock()


class TuneSpace(ctypes.Structure):
    _fields_ = [("bitmap_words", ctypes.POINTER(ctypes.c_uint32)), ("n_bitmap_words", ctypes.c_uint32),
                ("warps_per_block", ctypes.POINTER(ctypes.c_uint32)), ("n_warps_per_block", ctypes.c_uint32),
                ("unit_work", ctypes.POINTER(ctypes.c_uint32)), ("n_unit_work", ctypes.c_uint32),
                ("repeats", ctypes.c_uint32), ("occupancy", ctypes.POINTER(ctypes.c_uint32)),
                ("n_occupancy", ctypes.c_uint32)]


def cache_path() -> str:
    return os.environ.get("BBTC_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "bbtc_b200", "autotune.json"))


def gpu_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return f"cuda:{device}"


def graph_key(graph: core.Graph) -> str:
    st = graph.tile_stats()
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(graph.cuts, np.uint32).tobytes())
    h.update(st["nnz"].tobytes())
    return f"n={graph.n}|m={graph.m}|P={graph.P}|tiles={h.hexdigest()[:16]}"


def _arr(vals):
    a = (ctypes.c_uint32 * len(vals))(*vals)
    return a, len(vals)


def sweep(graph: core.Graph, base: core.Opts | None = None, bitmap_words=None, warps_per_block=None,
          unit_work=None, occupancy=None, repeats: int = 3) -> tuple[core.Opts, float]:
    """Run the library's sweep; returns the fastest options and their median ms."""
    lib = core.lib()
    lib.bbtc_autotune.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(TuneSpace),
                                  ctypes.POINTER(core.Opts), ctypes.POINTER(ctypes.c_double)]
    lib.bbtc_autotune.restype = ctypes.c_int
    o = core.Opts()
    if base is None:
        lib.bbtc_opts_default(ctypes.byref(o))
    else:
        ctypes.memmove(ctypes.byref(o), ctypes.byref(base), ctypes.sizeof(o))
    sp = TuneSpace()
    keep = []
    for field, vals in (("bitmap_words", bitmap_words), ("warps_per_block", warps_per_block),
                        ("unit_work", unit_work), ("occupancy", occupancy)):
        if vals:
            arr, n = _arr(list(vals))
            keep.append(arr)
            setattr(sp, field, ctypes.cast(arr, ctypes.POINTER(ctypes.c_uint32)))
            setattr(sp, "n_" + field, n)
    sp.repeats = repeats
    ms = ctypes.c_double()
    core.check(lib.bbtc_autotune(graph.ctx.handle, graph.handle, ctypes.byref(sp), ctypes.byref(o),
                                 ctypes.byref(ms)))
    return o, ms.value


def tune(graph: core.Graph, use_cache: bool = True, **kw) -> tuple[core.Opts, float | None]:
    """Cached autotune: returns (options, ms) -- ms is None on a cache hit."""
    key = f"{gpu_name(graph.ctx.device)}|{graph_key(graph)}"
    path = cache_path()
    if use_cache:
        with _lock:
            try:
                with open(path) as f:
                    hit = json.load(f).get(key)
            except (OSError, ValueError):
                hit = None
        if hit:
            o = core.options()
            for k, v in hit["opts"].items():
                setattr(o, k, v)
            return o, None
    o, ms = sweep(graph, **kw)
    if use_cache:
        with _lock:
            try:
                with open(path) as f:
                    data = json.load(f)
            except (OSError, ValueError):
                data = {}
            data[key] = {"opts": {f: getattr(o, f) for f, _ in core.Opts._fields_}, "ms": ms}
            os.makedirs(os.path.dirname(path), exist_ok=True)
            tmp = path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, path)
    return o, ms

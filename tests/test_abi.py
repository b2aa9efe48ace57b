"""The C-ABI library loads and exports every entry point include/bbtc_gpu.h
declares; calls that need no GPU behave (no compute is attempted here)."""
import ctypes
import os
import re

import numpy as np

from bbtc_b200 import _lib, core

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"^\s*(?:int|void)\s+(bbtc_\w+)\s*\(", src, flags=re.M)
    return names


def test_exports_every_declared_symbol():
    lib = ctypes.CDLL(os.path.join(_lib.LIBDIR, "libbbtc.so"))
    names = declared_functions()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_defaults():
    assert core.lib().bbtc_version() >= 10000
    o = core.options()
    assert o.mode == core.MODE_PERSISTENT and o.kernel == core.KERNEL_AUTO
    assert o.bitmap_words == 1024 and o.warps_per_block == 8 and o.use_cuda_graph == 1


def test_task_list_matches_reference_enumeration():
    for P in (1, 2, 3, 8, 16):
        t = core.task_list(P)
        want = [(i * P + j, j * P + k, i * P + k) for i in range(P) for j in range(i, P) for k in range(j, P)]
        assert [tuple(int(x) for x in r) for r in t] == want
        assert len(t) == P * (P + 1) * (P + 2) // 6


def test_errors_are_status_codes_not_crashes():
    lib = core.lib()
    h = ctypes.c_void_p()
    rc = lib.bbtc_ctx_create(0, ctypes.byref(h))
    if rc != 0:  # no GPU here
        assert rc == -6
        assert "device" in core.last_error().lower() or "cuda" in core.last_error().lower()
    else:
        lib.bbtc_ctx_destroy(h)
    assert lib.bbtc_task_list(0, None, 0, ctypes.byref(ctypes.c_uint32())) == -1
    assert lib.bbtc_task_list(65, None, 0, ctypes.byref(ctypes.c_uint32())) == -1
    assert lib.bbtc_graph_upload(None, 0, None, None, 0, None, 0, None) == -1
    assert lib.bbtc_count(None, None, None, 0, -1, None, None) == -1


def test_host_library_exports():
    lib = _lib.host()
    for n in ("bbtcg_rmat", "bbtcg_chung_lu", "bbtcg_rgg", "bbtcg_from_pairs", "bbtcp_cuts"):
        assert hasattr(lib, n)

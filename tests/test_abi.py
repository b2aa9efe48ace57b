"""The C-ABI library loads and exports every entry point include/bbtc_gpu.h
declares; calls that need no GPU behave (no compute is attempted here)."""
import ctypes
import os
import re

import numpy as np
import pytest

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
    assert o.bitmap_words == 0 and o.occupancy == 0  # resolved per request from the graphs' size
    assert o.warps_per_block == 8 and o.use_cuda_graph == 1


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
    out = ctypes.c_uint64()
    assert lib.bbtc_count_hybrid(None, None, None, None, None, 0, 0, 2, None, ctypes.byref(out), None) == -1
    assert "NULL" in core.last_error()


def test_allocation_fault_hook_arms_and_disarms():
    assert core.debug_fail_alloc(5) == -1
    assert core.debug_fail_alloc(2) == 5
    assert core.debug_fail_alloc(-1) == 2
    assert core.debug_fail_alloc(-1) == -1


@pytest.mark.parametrize("value,armed", [("3", 3), ("0", 0), ("abc", -1), ("-2", -1), ("", -1)])
def test_allocation_fault_hook_from_the_environment(value, armed):
    import subprocess
    import sys
    code = "from bbtc_b200 import core; print(core.debug_fail_alloc(-1))"
    env = dict(os.environ, BBTC_FAIL_ALLOC=value)
    out = subprocess.run([sys.executable, "-c", code], env=env, cwd=ROOT, capture_output=True, text=True,
                         timeout=120, check=True).stdout
    assert int(out.strip()) == armed


def test_cpp_mirror_reports_errors_as_exceptions(tmp_path):
    """include/bbtc.hpp (the reference's class names over the C ABI) turns a
    failing call into bbtc::Error with the status, where the reference would
    crash: here, a context on a machine without a usable GPU, and a task list
    for P outside [1, 64]."""
    import shutil
    import subprocess
    src = tmp_path / "mirror.cpp"
    src.write_text(r"""
#include <cstdio>
#include "bbtc.hpp"
int main() {
  int ctx_status = 0, list_status = 0;
  try { bbtc::Context ctx(0); } catch (const bbtc::Error& e) { ctx_status = e.status(); }
  try { bbtc::tasks::TaskList(65); } catch (const bbtc::Error& e) { list_status = e.status(); }
  std::printf("%d %d %zu\n", ctx_status, list_status, bbtc::tasks::TaskList(4).size());
  (void)&bbtc::BBTc::SetCpuWorkers;  // the hybrid methods compile
  (void)&bbtc::BBTc::LastHybridStats;
  return 0;
}
""")
    exe = tmp_path / "mirror"
    cxx = shutil.which("g++") or shutil.which("c++")
    subprocess.run([cxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe),
                    "-L", _lib.LIBDIR, "-lbbtc", "-Wl,-rpath," + _lib.LIBDIR], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True, timeout=120).stdout.split()
    ctx_status, list_status, n4 = (int(x) for x in out)
    assert ctx_status in (0, -6)  # -6: no usable device here; 0 where a B200 is present
    assert list_status == -1 and n4 == 20


def test_host_library_exports():
    lib = _lib.host()
    for n in ("bbtcg_rmat", "bbtcg_chung_lu", "bbtcg_rgg", "bbtcg_from_pairs", "bbtcp_cuts"):
        assert hasattr(lib, n)


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes mirror has the size and field offsets gcc gives the C struct."""
    import shutil
    import subprocess
    from bbtc_b200 import autotune
    mirrors = {"bbtc_task": core.Task, "bbtc_opts": core.Opts, "bbtc_graph_info": core.GraphInfo,
               "bbtc_tune_space": autotune.TuneSpace, "bbtc_csr_dev": core.CsrDev,
               "bbtc_server_opts": core.ServerOpts, "bbtc_request_info": core.RequestInfo,
               "bbtc_server_stats": core.ServerStats, "bbtc_hybrid_stats": core.HybridStats}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "bbtc_gpu.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    cc = shutil.which("gcc") or shutil.which("cc")
    subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])

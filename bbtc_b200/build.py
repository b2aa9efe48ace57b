"""Build the in-tree libraries and the CLI.

  lib/libbbtc.so       CUDA path + C ABI (include/bbtc_gpu.h), sm_100a only
  lib/libbbtc_host.so  graph generators and partitioners (host, OpenMP)
  bin/bbtc             drop-in CLI for the reference's `bbtc` executable

Run `python -m bbtc_b200.build` (or `__graft_entry__.build()`).  nvcc
cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("BBTC_CXX", shutil.which("g++") or "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["api.cu", "layout.cu", "count.cu", "server.cu", "prep.cu", "partition_dev.cu", "hybrid.cpp"]
HOST_SOURCES = ["graphgen.cpp", "partition.cpp", "graph_io.cpp"]


def _run(cmd: list[str]) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(names: list[str]) -> list[str]:
    extra = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh", ".hpp"))]
    return [os.path.join(CSRC, n) for n in names] + extra + [os.path.join(ROOT, "include", "bbtc_gpu.h")]


def build_host(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libbbtc_host.so")
    deps = _deps(HOST_SOURCES)
    if force or _stale(out, deps):
        _run([CXX, "-O3", "-march=x86-64-v2", "-fopenmp", "-std=c++17", "-shared", "-fPIC", "-o", out]
             + [os.path.join(CSRC, s) for s in HOST_SOURCES])
    return out


def build_cuda(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    out = os.path.join(LIB, "libbbtc.so")
    deps = _deps(CUDA_SOURCES)
    if force or _stale(out, deps):
        flags = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                 "-Xcompiler", "-O3", "-shared"] + ARCH
        if verbose_ptxas:
            flags += ["-Xptxas", "-v"]
        _run([NVCC] + flags + ["-o", out] + [os.path.join(CSRC, s) for s in CUDA_SOURCES])
    return out


def build_cli(force: bool = False) -> str | None:
    src = os.path.join(CSRC, "bbtc_cli.cpp")
    if not os.path.exists(src):
        return None
    os.makedirs(BIN, exist_ok=True)
    out = os.path.join(BIN, "bbtc")
    deps = _deps(["bbtc_cli.cpp"] + HOST_SOURCES)
    deps = [d for d in deps if os.path.exists(d)]
    if force or _stale(out, deps + [os.path.join(LIB, "libbbtc.so")]):
        srcs = [os.path.join(CSRC, s) for s in ["bbtc_cli.cpp"] + HOST_SOURCES
                if os.path.exists(os.path.join(CSRC, s))]
        _run([CXX, "-O3", "-fopenmp", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", out] + srcs
             + ["-L", LIB, "-lbbtc", "-Wl,-rpath,$ORIGIN/../lib", "-L/usr/local/cuda/lib64", "-lcudart"])
    return out


def build_all(force: bool = False) -> None:
    build_host(force)
    build_cuda(force)
    build_cli(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)

"""bench.py's reference arm on the CPU: one JSON line with the contract's
keys, printed by rank 0 alone when launched as two ranks (gloo, 127.0.0.1)."""
import json
import os
import socket
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = ["--impl", "reference", "--scale", "12", "--ncut", "8", "--steps", "2", "--warmup", "1"]

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


def _lines(out):
    return [json.loads(l) for l in out.splitlines() if l.startswith("{")]


def _check(res, world):
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in res, k
    assert res["impl"] == "reference" and res["n_gpus"] == world and res["steps"] == 2 and res["warmup"] == 1
    assert res["value"] > 0 and res["unit"] == "edges/s" and res["higher_is_better"] is True
    cb = res["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == res["value"] and cb["sample"]
    assert res["e2e"] == {"value": res["value"], "unit": res["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}


def test_reference_arm_one_process():
    out = subprocess.run([sys.executable, "bench.py", *ARGS], cwd=ROOT, capture_output=True, text=True,
                         timeout=300, check=True).stdout
    lines = _lines(out)
    assert len(lines) == 1
    _check(lines[0], 1)


def test_reference_arm_two_ranks_prints_once():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py", *ARGS]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = _lines(r.stdout)
    assert len(lines) == 1
    _check(lines[0], 2)

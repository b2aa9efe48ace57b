"""The drop-in `bbtc` executable: flags and messages as in the reference
(include/utils/utils.hpp:50-154).  Runs without a GPU: every case here exits
during argument checking."""
import os
import subprocess

import pytest

from bbtc_b200 import build

EXE = os.path.join(os.path.dirname(build.__file__), "bin", "bbtc")


def run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=60)


@pytest.fixture(scope="module", autouse=True)
def _cli():
    build.build_cli()


def test_usage_on_too_few_arguments():
    r = run("--help")
    assert r.returncode == 0 and "syntax: bbtc --graph <path> [OPTION].. [--help]" in r.stdout


def test_wrong_argument(tmp_path):
    g = tmp_path / "g.el"
    g.write_text("0 1\n")
    r = run("--graph", str(g), "--bogus")
    assert "Wrong argument '--bogus' given." in r.stdout and r.returncode == 0


def test_missing_graph():
    r = run("--graph", "/nonexistent/graph.el", "--ncut", "4")
    assert "Graph doesn't exist" in r.stdout


def test_range_checks(tmp_path):
    g = tmp_path / "g.el"
    g.write_text("0 1\n")
    assert "--ncut has to be set in between: 1 < --ncut < 65" in run("--graph", str(g), "--ncut", "1").stdout
    assert "--repeat has to be set in between: 0 < --repeat" in run("--graph", str(g), "--repeat", "0").stdout
    assert "--border has to be set in between: -2 < --border" in run("--graph", str(g), "--border", "-3").stdout
    assert "Wrong partitioning algorithm." in run("--graph", str(g), "--partitioner", "xyz").stdout


def test_cpu_workers_flag_bounds(tmp_path):
    """--cpu-workers (not in the reference) takes -1 (the reference's split of
    OpenMP threads) and up; below that the range message and usage, exit 0."""
    g = tmp_path / "g.el"
    g.write_text("0 1\n")
    r = run("--graph", str(g), "--cpu-workers", "-2")
    assert "--cpu-workers has to be set in between: -2 < --cpu-workers" in r.stdout and r.returncode == 0
    assert "--cpu-workers <int>" in run("--help").stdout
    for v in ("-1", "0", "6"):
        r = run("--graph", str(g), "--cpu-workers", v, "--border", "3")
        assert "has to be set in between" not in r.stdout, v

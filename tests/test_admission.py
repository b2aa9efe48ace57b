"""The request server's admission policy (bbtc_b200/csrc/admission.hpp),
compiled on its own with the host C++ compiler: smallest first, the oldest
first once it has waited long enough, the HBM budget, loaders reserved for
small requests."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include <vector>
#include "admission.hpp"
struct R { uint64_t m, reserved, t_submit; };
static long pick(std::vector<R>& rs, uint64_t budget, uint64_t in_use, uint64_t now, bool small_only,
                 bool large_ok = true, uint64_t small_aging = 0) {
  std::vector<const R*> p;
  for (auto& r : rs) p.push_back(&r);
  bbtc::AdmitLimits lim{budget, in_use, /*small_edges=*/1000, /*aging_ns=*/50, now, small_only, 4096};
  lim.large_ok = large_ok;
  lim.small_aging_ns = small_aging;
  const size_t i = bbtc::admit_pick(p, lim);
  return i == SIZE_MAX ? -1 : (long)i;
}
int main() {
  std::vector<R> a{{500, 10, 0}, {20, 10, 5}, {300, 10, 6}};
  std::printf("smallest %ld\n", pick(a, 1000, 0, 10, false));        // 1: fewest edges
  std::printf("aged %ld\n", pick(a, 1000, 0, 60, false));            // 0: waited >= 50
  std::vector<R> b{{20, 600, 0}, {30, 100, 1}};
  std::printf("budget %ld\n", pick(b, 1000, 500, 10, false));        // 1: 500 + 600 > 1000
  std::printf("empty_device %ld\n", pick(b, 1000, 0, 10, false));    // 0: nothing held, anything fits
  std::vector<R> c{{20, 2000, 0}};
  std::printf("never_fits %ld\n", pick(c, 1000, 900, 10, false));    // 0: taken, to fail at once
  std::vector<R> d{{5000, 10, 0}, {4000, 10, 1}};
  std::printf("small_only %ld\n", pick(d, 1000, 0, 10, true));       // -1: both are large
  std::printf("any_loader %ld\n", pick(d, 1000, 0, 10, false));      // 1
  std::printf("large_busy %ld\n", pick(d, 1000, 0, 60, false, false)); // -1: large loads at their limit, even aged
  std::vector<R> f{{5000, 10, 0}, {40, 10, 1}};
  std::printf("small_while_large %ld\n", pick(f, 1000, 0, 60, false, false)); // 1
  std::vector<R> g{{5000, 10, 0}, {800, 10, 2}, {40, 10, 9}};
  std::printf("small_not_aged %ld\n", pick(g, 1000, 0, 10, false, true, 20));  // 2: fewest edges
  std::printf("small_aged %ld\n", pick(g, 1000, 0, 30, false, true, 20));      // 1: small, waited >= 20
  std::printf("large_aged_first %ld\n", pick(g, 1000, 0, 60, false, true, 20)); // 0: the oldest aged
  std::vector<R> e;
  std::printf("none %ld\n", pick(e, 1000, 0, 10, false));            // -1
  return 0;
}
"""


def test_admission_policy(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "admit.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "admit"
    subprocess.run([cxx, "-std=c++17", "-I", os.path.join(ROOT, "bbtc_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], check=True, capture_output=True,
                                                 text=True).stdout.splitlines())
    assert out == {"smallest": "1", "aged": "0", "budget": "1", "empty_device": "0", "never_fits": "0",
                   "small_only": "-1", "any_loader": "1", "none": "-1", "large_busy": "-1",
                   "small_while_large": "1", "small_not_aged": "2", "small_aged": "1",
                   "large_aged_first": "0"}

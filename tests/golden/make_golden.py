"""Generate tests/golden/*.npz: small graphs and the counts the reference's own
code gives for them.

Run in a container that has the reference tree (oracle/_ref built from it):
    python tests/golden/make_golden.py          # everything
    python tests/golden/make_golden.py --rac    # sarma-rac-cuts.npz only
Each fixture holds the oriented CSR (indptr, indices), and for every cut vector
(`cuts_<part>_<P>`) the count of the reference's CPU path compiled from its
sources (oracle.ref_count).  `cli_triangles` / `cli_edges` come from the
reference's unmodified executable run on the graph as an edge list (its own
reader, symmetriser, degree order and SARMA pal cuts, ncut 4).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from bbtc_b200 import graphs  # noqa: E402


def pairs(n, edges, name):
    return graphs.from_pairs(n, [a for a, _ in edges], [b for _, b in edges], name=name)


def cases():
    yield graphs.rmat(8, 8, seed=1)
    yield graphs.rmat(10, 16, seed=2)
    yield graphs.rmat(11, 32, seed=3)
    yield graphs.rgg(1 << 11, seed=4)
    yield graphs.chung_lu(1 << 12, seed=5, max_deg=300)
    n = 20
    yield pairs(n, [(a, b) for a in range(n) for b in range(a + 1, n)], "complete-20")
    w = 30
    yield pairs(w + 1, [(0, i) for i in range(1, w + 1)] + [(i, i % w + 1) for i in range(1, w + 1)], "wheel-30")
    yield pairs(25, [(a, b) for a in range(10) for b in range(10, 25)], "bipartite-10-15")
    yield pairs(36, [(r * 6 + c, r * 6 + c + 1) for r in range(6) for c in range(5)]
                + [(r * 6 + c, (r + 1) * 6 + c) for r in range(5) for c in range(6)], "grid-6x6")
    yield pairs(3, [(0, 1), (1, 2), (0, 2)], "triangle")


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built; run `make -C oracle` with the reference tree present")
    for g in cases():
        out = {"n": np.uint32(g.n), "indptr": g.indptr, "indices": g.indices}
        for part in ("uni", "n1d", "pal"):
            for P in (1, 4, 8):
                cuts = graphs.cuts(g, P, part)
                ref, _ = oracle.ref_count(g.n, g.indptr, g.indices, cuts, nthreads=4)
                out[f"cuts_{part}_{P}"] = cuts
                out[f"count_{part}_{P}"] = np.uint64(ref)
        if g.m:
            cli = oracle.ref_cli(g.n, g.indptr, g.indices, "pal", 4, nthreads=4)
            out["cli_triangles"] = np.uint64(cli["triangles"])
            out["cli_edges"] = np.uint64(cli["edges"])
        path = os.path.join(HERE, f"{g.name}.npz")
        np.savez_compressed(path, **out)
        print(f"{g.name}: n={g.n} m={g.m} triangles={int(out['count_uni_1'])}")


# Graphs whose rac cuts are pinned (sarma-rac-cuts.npz): regenerated from
# these calls by the test, so only the cut vectors are stored.
RAC_CASES = {
    "rmat-s12-ef16-seed3": lambda: graphs.rmat(12, 16, seed=3),
    "rmat-s14-ef8-seed5": lambda: graphs.rmat(14, 8, seed=5),
    "chunglu-n8192-seed6": lambda: graphs.chung_lu(1 << 13, seed=6, max_deg=400.0),
}
RAC_P = (3, 8, 16, 33)


def _ref_rac_child(key, P):
    g = RAC_CASES[key]()
    print(" ".join(str(int(c)) for c in oracle.ref_cuts(g.n, g.indptr, g.indices, P, "rac")))


def rac_main():
    """SARMA's rac cuts (refine_a_cut::partition, the reference's call
    sequence in oracle/_ref) for RAC_CASES x RAC_P.  Each runs in a child
    process, retried: SARMA's parallel loops crashed the process now and then
    (a segmentation fault inside the reference's code, not reproducible on
    its own)."""
    import subprocess
    out = {}
    for key in RAC_CASES:
        for P in RAC_P:
            for attempt in range(5):
                r = subprocess.run([sys.executable, os.path.abspath(__file__), "--rac-child", key, str(P)],
                                   capture_output=True, text=True)
                if r.returncode == 0:
                    break
            else:
                raise SystemExit(f"SARMA rac failed for {key} P={P}: {r.stderr[-300:]}")
            out[f"{key}__{P}"] = np.array([int(x) for x in r.stdout.split()], dtype=np.uint32)
            print(key, P, "attempts", attempt + 1)
    np.savez_compressed(os.path.join(HERE, "sarma-rac-cuts.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--rac-child":
        _ref_rac_child(sys.argv[2], int(sys.argv[3]))
    elif len(sys.argv) > 1 and sys.argv[1] == "--rac":
        rac_main()
    else:
        main()
        rac_main()

#!/usr/bin/env python
"""Benchmark: exact triangle counting, edges/s, on B200.

Workload (N=1): R-MAT scale 22, edge factor 16, a/b/c/d = .57/.19/.19/.05,
seed 2, symmetrised / deduplicated / degree-ordered and oriented, pal cuts,
ncut 16 -- the single-graph B200 configuration.  A step is one exact count of
the whole graph (every task of TaskList(16)).

  value  persistent form, graph resident in HBM, device time of the count
         (CUDA events on the library's stream), edges / second
  plain  the same count as one launch per task (reported beside it)
  e2e    the public C ABI from pinned host buffers: CSR upload + device layout
         build + count + result readback, every step, wall clock
  roofline  B_alg = 4 m + 4 sum_{(u,v)} (d+(u) + d+(v)) bytes per count over
         the count's device time, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own CPU path (oracle/_ref, built from its
         sources) on the box's host cores, same graph and cuts

`--impl reference` times only the reference's CPU path (all host threads).
For N > 1 (torchrun) every rank counts its own graph of the same shape
(seed 2 + rank): weak scaling, no collective on the data path; the counts are
summed with one all_reduce after the timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

# one hardware work queue per stream (the serving mode runs ten or more);
# read when the process initialises CUDA, so set before torch is imported
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges/sec at exact count, batched vs plain form on 1 B200; p50/p99 latency"
UNIT = "edges/s"
FALLBACK_HBM_GBS = 6650.0
# serving throughput peak on one B200: requests/s served when the offered
# rate exceeds what the server sustains, with the server's default
# configuration (1,800 req/s offered for 30 s: 1,450 and 1,454 served,
# 4.44e9-4.45e9 edges/s, two runs); the default line serves at 80 % of it
SERVE_PEAK_RPS = 1450.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=int, default=22)
    p.add_argument("--family", default="rmat", choices=["rmat", "chunglu"],
                   help="rmat (default) or chunglu (n = 2^scale; the 8M-vertex n1d ncut 32 case is "
                        "--family chunglu --scale 23 --seed 3 --partitioner n1d --ncut 32)")
    p.add_argument("--edge-factor", type=int, default=16)
    p.add_argument("--seed", type=int, default=2)
    p.add_argument("--ncut", type=int, default=16)
    p.add_argument("--partitioner", default="pal")
    p.add_argument("--kernel", default="auto")
    p.add_argument("--bitmap-words", type=int, default=0)
    p.add_argument("--unit-work", type=int, default=0)
    p.add_argument("--occupancy", type=int, default=0)
    p.add_argument("--warps", type=int, default=0)
    p.add_argument("--no-autotune", action="store_true",
                   help="skip the launch-option sweep (bbtc_autotune) that picks the headline's bitmap size and "
                        "register budget; explicit --bitmap-words / --occupancy also skip it")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--cpu-threads", type=int, default=0)
    p.add_argument("--config", default="single", choices=["single", "batch", "serve", "hybrid"],
                   help="single: one R-MAT s22 graph (default); batch: 512 R-MAT + 64 RGG graphs in one "
                        "launch; serve: Poisson request stream through the continuous-batching server; "
                        "hybrid: the graph counted by the GPU and CPU workers together (bbtc_count_hybrid)")
    p.add_argument("--border", type=int, default=0, help="hybrid: the reference's --border (default 0)")
    p.add_argument("--cpu-workers", type=int, default=0,
                   help="hybrid: CPU worker threads (0: one per host core but one)")
    p.add_argument("--batch-max-scale", type=int, default=20)
    p.add_argument("--batch-plain-steps", type=int, default=-1,
                   help="batch: steps of the one-launch-per-task comparison (-1: steps / 2, at least 2)")
    p.add_argument("--rate", type=float, default=600.0, help="serve: requests per second")
    p.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals")
    p.add_argument("--serve-max-scale", type=int, default=22)
    p.add_argument("--loaders", type=int, default=6, help="serve: loader threads")
    p.add_argument("--pin", type=int, default=1, help="serve: request buffers in page-locked host memory")
    p.add_argument("--copy-engine-uploads", action="store_true",
                   help="serve: small requests go through the copy engines even from page-locked buffers")
    p.add_argument("--trace", default="", help="serve: write every request's stage timestamps to this JSON file")
    p.add_argument("--rates", default="", help="serve: comma-separated rates, one stream each on one server")
    p.add_argument("--large-bps", type=int, default=0, help="serve: persistent blocks per SM of the large lane (0: 3)")
    p.add_argument("--large-layout-bps", type=int, default=0,
                   help="serve: layout blocks per SM of large requests (0: 2)")
    p.add_argument("--small-sms", type=int, default=-1,
                   help="serve: SMs of the small requests' partition (0: none; -1: the server's default)")
    p.add_argument("--max-large-loads", type=int, default=-1,
                   help="serve: large requests loading at once (0: no limit; -1: the server's default)")
    p.add_argument("--small-aging-us", type=int, default=-1,
                   help="serve: a small request waiting this long is loaded before smaller ones "
                        "(0: the large requests' aging; -1: the server's default)")
    p.add_argument("--no-check", action="store_true", help="batch / serve: skip the oracle counts")
    p.add_argument("--no-batch", action="store_true", help="default line: no batched-launch sub-record")
    p.add_argument("--no-serve", action="store_true", help="default line: no serving sub-record")
    p.add_argument("--no-hybrid", action="store_true", help="default line: no hybrid GPU + CPU sub-record")
    p.add_argument("--sub-batch-max-scale", type=int, default=14,
                   help="default line: largest R-MAT scale of the batched-launch sub-record")
    p.add_argument("--sub-serve-rate", type=float, default=0.0,
                   help="default line: serving rate (0: 80 %% of SERVE_PEAK_RPS)")
    p.add_argument("--sub-serve-duration", type=float, default=10.0)
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """Samples the SM clock and the clock-event reasons every 5 ms through NVML
    (read-only queries) while the timed region runs; nvidia-smi (200 ms) when
    NVML is not importable."""

    NAMES = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.thread = None
        self.samples = []
        self.smax = None
        self.reason_bits = 0
        self.stop_flag = threading.Event()

    def _handle(self, nv):
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.device)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.nv, self.h = nv, h
            self.smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons",
                                  getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons", None))

            def run():
                while not self.stop_flag.is_set():
                    try:
                        self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        if get_reasons is not None:
                            self.reason_bits |= get_reasons(h)
                    except Exception:
                        pass
                    time.sleep(0.005)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join()
            reasons = sorted(k for k, attr in self.NAMES.items()
                             if self.reason_bits & getattr(self.nv, attr, 0))
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass
            return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(self.samples), "source": "nvml, 5 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [ln.strip().split(",") for ln in self.file.read().splitlines() if ln.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = list(self.NAMES)
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def load_traffic(family: str, scale: int, ncut: int):
    """Per-launch DRAM bytes of the count kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_fused_queue_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        key = f"{family}-s{scale}-p{ncut}"
        return d[key]["dram_bytes_per_launch"], d[key].get("note")
    except Exception:
        return None, None


def workload_name(args) -> str:
    if args.family == "chunglu":
        return f"chunglu-n{1 << args.scale}-g2.1-mean20-cap50000-seed{args.seed}"
    return f"rmat-s{args.scale}-ef{args.edge_factor}-seed{args.seed}"


def make_graph(args, seed):
    from bbtc_b200 import graphs
    t0 = time.time()
    if args.family == "chunglu":
        # Chung-Lu, n = 2^scale, gamma 2.1, mean degree 20, weights capped at 50,000
        g = graphs.chung_lu(1 << args.scale, 2.1, 20.0, 50000.0, seed=seed)
    else:
        g = graphs.rmat(args.scale, args.edge_factor, seed=seed)
    cuts = graphs.cuts(g, args.ncut, args.partitioner)
    return g, cuts, time.time() - t0


def reference_graph(args, seed):
    """The benchmark graph and the reference's own cut vector, from oracle/
    code only: the generators' restatement (oracle/graphs_oracle.c, bit-equal
    to the library's) and the reference's SARMA partitioner (oracle/_ref)."""
    import oracle
    t0 = time.time()
    if args.family == "chunglu":
        n, indptr, indices = oracle.chung_lu(1 << args.scale, 2.1, 20.0, 50000.0, seed=seed)
    else:
        n, indptr, indices = oracle.rmat(args.scale, args.edge_factor, seed=seed)
    part = "pal" if args.partitioner.startswith("pal") else args.partitioner
    cuts = oracle.ref_cuts(n, indptr, indices, args.ncut, part)
    return n, indptr, indices, cuts, time.time() - t0


def run_reference(args, rank: int):
    """Reference arm: the reference's own CPU counting path on all host
    threads, fed the same graph (generated by the oracle's restatement) and
    cut by the reference's own SARMA partitioner; nothing of this library is
    loaded."""
    import oracle
    if rank != 0:
        return None
    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libbbtc_ref.so not built"}
    n, indptr, indices, cuts, gen_s = reference_graph(args, args.seed)
    m = int(indices.shape[0])
    threads = args.cpu_threads or os.cpu_count()
    count, secs = oracle.ref_count(n, indptr, indices, cuts, nthreads=threads, repeat=args.warmup + args.steps)
    timed = secs[args.warmup:]
    t = statistics.median(timed)
    value = m / t
    sample = (f"full workload per step: NoOfTriangles() over all {args.ncut * (args.ncut + 1) * (args.ncut + 2) // 6}"
              f" tasks, median of {len(timed)} steps after {args.warmup} warm-up")
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "device": "host cores (rank 0 only)", "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"{workload_name(args)} {args.partitioner} ncut {args.ncut}", "n": n, "m": m,
                   "P": args.ncut, "partitioner": args.partitioner, "triangles": count,
                   "cuts": "the reference's SARMA partitioner (include/utils/utils.hpp:271-288)",
                   "graph": "oracle/graphs_oracle.c (the generators' restatement)", "generate_s": round(gen_s, 2)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def batch_workload(max_scale: int):
    """512 R-MAT graphs (scale uniform in [10, max_scale], edge factor uniform
    in 8..32) and 64 random geometric graphs (2^14..2^18 points, mean degree
    12), seeds 100..675 in order, each with its own uni ncut in 4..16."""
    from bbtc_b200 import graphs
    rng = np.random.default_rng(12345)
    out = []
    for i in range(512):
        seed = 100 + i
        s = int(rng.integers(10, max_scale + 1))
        ef = int(rng.integers(8, 33))
        P = int(rng.integers(4, 17))
        out.append((graphs.rmat(s, ef, seed=seed), P))
    for i in range(64):
        seed = 612 + i
        n = int(round(2 ** rng.uniform(14, 18)))
        P = int(rng.integers(4, 17))
        out.append((graphs.rgg(n, mean_deg=12.0, seed=seed), P))
    return [(g, graphs.cuts(g, P, "uni")) for g, P in out]


def oracle_counts(items, threads: int = 0):
    """The oracle's count of every (graph, cuts) pair (the C restatement of
    the reference's CPU path), largest graphs first."""
    import oracle
    order = sorted(range(len(items)), key=lambda i: -items[i][0].m)
    out = [None] * len(items)
    for i in order:
        g, c = items[i]
        out[i] = oracle.count(g.n, g.indptr, g.indices, c, nthreads=threads)
    return out


def measure_batch(ctx, max_scale: int, steps: int, warmup: int, plain_steps: int, check: bool = True) -> dict:
    """The batched launch: every graph of the batch workload in one persistent
    launch (bbtc_count_batch), against each graph counted alone with one
    launch per task.  With `check`, every graph's count is first compared
    with the oracle's."""
    import torch
    from bbtc_b200 import Graph, count_batch, options
    t0 = time.time()
    work = batch_workload(max_scale)
    gen_s = time.time() - t0
    t0 = time.time()
    want = oracle_counts(work) if check else None
    oracle_s = time.time() - t0
    sts = [Graph.from_csr(ctx, g, c) for g, c in work]
    try:
        m_total = sum(g.m for g, _ in work)
        po = options(mode="persistent")
        first = count_batch(ctx, sts, po)
        if check:
            bad = [i for i, (a, b) in enumerate(zip(first, want)) if a != b]
            assert not bad, f"batch counts differ from the oracle for graphs {bad[:8]}"
        for _ in range(warmup):
            assert count_batch(ctx, sts, po) == first
        ts = []
        for _ in range(steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            got = count_batch(ctx, sts, po)
            ts.append(time.perf_counter() - t)
            assert got == first
        plain = options(mode="plain", cuda_graph=False)
        pts = []
        for _ in range(plain_steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            got = [st.count(opts=plain) for st in sts]
            pts.append(time.perf_counter() - t)
            assert got == first
    finally:
        for st in sts:
            st.free()
    tb = statistics.median(ts)
    res = {"value": m_total / tb, "unit": UNIT, "ms_per_step": tb * 1e3, "steps": steps,
           "workload": f"512 R-MAT s10-{max_scale} ef 8-32 + 64 RGG 2^14-2^18, seeds 100-675, uni ncut 4-16",
           "graphs": len(work), "m_total": m_total, "triangles_total": int(sum(first)),
           "oracle_checked": bool(check), "generate_s": round(gen_s, 1), "oracle_s": round(oracle_s, 1),
           "timing": "wall clock of bbtc_count_batch (plan + one persistent launch + readback)"}
    if pts:
        tp = statistics.median(pts)
        res["plain"] = {"value": m_total / tp, "ms_per_step": tp * 1e3,
                        "note": "every graph counted alone, one launch per task", "batched_over_plain": tp / tb}
    return res


def run_batch(args):
    from bbtc_b200 import Context
    ctx = Context(0)
    plain_steps = args.batch_plain_steps if args.batch_plain_steps >= 0 else max(2, args.steps // 2)
    b = measure_batch(ctx, args.batch_max_scale, args.steps, args.warmup, plain_steps, check=not args.no_check)
    ctx.close()
    res = {"metric": METRIC, "value": b.pop("value"), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": b.pop("ms_per_step"), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32", "data": "synthetic",
           "config": {"workload": "batch: " + b.pop("workload"), **{k: v for k, v in b.items() if k != "plain"}},
           "plain": b.get("plain")}
    print(json.dumps(res), flush=True)


def run_hybrid(args):
    """bbtc_count_hybrid on one graph: the reference's default border 0, one CPU
    worker per host core but one beside the GPU; wall clock per call, the
    host CSR's row checks included."""
    from bbtc_b200 import Context, Graph, options
    ctx = Context(0)
    g, cuts, _ = make_graph(args, args.seed)
    st = Graph.from_csr(ctx, g, cuts)
    want = st.count()
    workers = args.cpu_workers if args.cpu_workers > 0 else max(1, (os.cpu_count() or 2) - 1)
    tl = st.task_list(sorted=True)
    ho = options(mode="persistent", kernel="bitmap", bitmap_words=args.bitmap_words, cuda_graph=False)
    ht, hs = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        hc, hstat = st.count_hybrid(g.indptr, g.indices, tl, args.border, workers, ho)
        t1 = time.perf_counter()
        assert hc == want, f"hybrid count disagrees: {hc} vs {want}"
        if i >= args.warmup:
            ht.append(t1 - t0)
            hs.append(hstat)
    th = statistics.median(ht)
    st.free()
    ctx.close()
    res = {"metric": METRIC, "value": g.m / th, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": th * 1e3, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "u32", "data": "synthetic",
           "config": {"workload": f"hybrid: {workload_name(args)} {args.partitioner} ncut {args.ncut}",
                      "border": args.border, "cpu_workers": workers, "triangles": want,
                      "gpu_side": "per-task persistent queue (bitmap kernel) over contiguous ranges from the head"},
           "splits": [{k: h[k] for k in ("gpu_tasks", "cpu_tasks", "gpu_launches", "separator")} for h in hs],
           "gpu_ms": [h["gpu_ms"] for h in hs], "cpu_ms": [h["cpu_ms"] for h in hs],
           "note": "wall clock of bbtc_count_hybrid (CPU workers from the tail of the sorted list, the GPU from "
                   "the head), median over the steps; every count equal to the GPU-only count"}
    print(json.dumps(res), flush=True)


def serve_pool(max_scale: int, pin: bool):
    """Request graphs: R-MAT scale 12 + Geom(0.3) truncated at max_scale, edge
    factor 16; a pool of distinct seeds per scale (fewer for the big ones).
    With `pin`, the CSRs sit in page-locked host memory, as a serving front
    end that receives requests into pinned buffers holds them."""
    import types
    from bbtc_b200 import graphs
    keep = []

    def pinned(a):
        import torch
        t = torch.empty(max(1, a.size), dtype=torch.int32, pin_memory=True)
        t.numpy()[:a.size] = a.view(np.int32)
        keep.append(t)
        return t.numpy()[:a.size].view(np.uint32)

    pool = {}
    for s in range(12, max_scale + 1):
        k = 8 if s <= 16 else (4 if s <= 19 else 2)
        gs = []
        for j in range(k):
            g = graphs.rmat(s, 16, seed=10000 + 100 * s + j)
            c = graphs.cuts(g, 4 if s < 16 else 8, "pal")
            if pin:
                g = types.SimpleNamespace(n=g.n, m=g.m, indptr=pinned(g.indptr), indices=pinned(g.indices))
            gs.append((g, c))
        pool[s] = gs
    return pool, keep


def serve_once(srv, pool, max_scale: int, rate: float, duration: float, seed: int, want=None, trace=None) -> dict:
    """One Poisson request stream through the server: `rate` requests/s for
    `duration` s; latency is bbtc_submit -> count in host memory.  `want`
    maps (scale, index) to the oracle's count of that pool graph."""
    import threading
    rng = np.random.default_rng(seed)
    n_req = max(1, int(rate * duration))
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    scales = np.minimum(12 + rng.geometric(0.3, size=n_req) - 1, max_scale)
    which = [int(rng.integers(len(pool[int(s)]))) for s in scales]
    ids = [None] * n_req
    start = time.perf_counter()

    def submitter():
        for i in range(n_req):
            delay = arrivals[i] - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            g, c = pool[int(scales[i])][which[i]]
            ids[i] = srv.submit_csr(g, c)

    th = threading.Thread(target=submitter)
    th.start()
    lat, lat18, edges, first_sub, last_done = [], [], 0, None, 0
    stages = {"queue": [], "load": [], "ready_wait": [], "count": []}
    by_scale = {}
    checked = 0
    for i in range(n_req):
        while ids[i] is None:
            time.sleep(0.0002)
        info = srv.wait(ids[i])
        assert info.status == 1, info.status
        key = (int(scales[i]), which[i])
        if want is not None:
            assert info.count == want[key], (key, info.count, want[key])
            checked += 1
        ms = (info.done_ns - info.submit_ns) / 1e6
        lat.append(ms)
        stages["queue"].append((info.load_ns - info.submit_ns) / 1e6)
        stages["load"].append((info.ready_ns - info.load_ns) / 1e6)
        stages["ready_wait"].append((info.launch_ns - info.ready_ns) / 1e6)
        stages["count"].append((info.done_ns - info.launch_ns) / 1e6)
        if scales[i] <= 18:
            lat18.append(ms)
        by_scale.setdefault(int(scales[i]), []).append(
            (ms, (info.ready_ns - info.load_ns) / 1e6, (info.done_ns - info.launch_ns) / 1e6))
        if trace is not None:
            trace.append((int(scales[i]), int(pool[key[0]][key[1]][0].m), info.submit_ns, info.load_ns,
                          info.ready_ns, info.launch_ns, info.done_ns, info.batch))
        edges += pool[key[0]][key[1]][0].m
        first_sub = info.submit_ns if first_sub is None else min(first_sub, info.submit_ns)
        last_done = max(last_done, info.done_ns)
        srv.release(ids[i])
    th.join()
    span = (last_done - first_sub) / 1e9
    return {"rate": rate, "duration_s": duration, "requests": n_req, "value": edges / span, "unit": UNIT,
            "requests_per_s": n_req / span, "oracle_checked": checked,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "p50_scale_le_18": float(np.percentile(lat18, 50)) if lat18 else None,
                           "p99_scale_le_18": float(np.percentile(lat18, 99)) if lat18 else None,
                           "n_scale_le_18": len(lat18),
                           "definition": "bbtc_submit -> count in host memory (server steady clock)"},
            "stages_ms_p50_p99": {k: [float(np.percentile(v, 50)), float(np.percentile(v, 99))]
                                  for k, v in stages.items()},
            "by_scale_p50_ms": {s: {"n": len(v), "latency": float(np.percentile([x[0] for x in v], 50)),
                                    "load": float(np.percentile([x[1] for x in v], 50)),
                                    "count": float(np.percentile([x[2] for x in v], 50))}
                                for s, v in sorted(by_scale.items())}}


def measure_serve(max_scale: int, rates, duration: float, loaders: int, pin: bool, copy_engine_uploads: bool,
                  check: bool = True, trace=None, large_bps: int = 0, large_layout_bps: int = 0,
                  max_large_loads: int = -1, small_sms: int = -1, small_aging_us: int = -1) -> dict:
    """Pool generation, oracle counts of every pool graph, one warm-up
    request per scale, then one Poisson stream per rate on the same server."""
    from bbtc_b200 import Server
    t0 = time.time()
    pool, keep = serve_pool(max_scale, pin)
    gen_s = time.time() - t0
    t0 = time.time()
    want = None
    if check:
        items = [(g, c) for s in sorted(pool) for g, c in pool[s]]
        keys = [(s, j) for s in sorted(pool) for j in range(len(pool[s]))]
        want = dict(zip(keys, oracle_counts(items)))
    oracle_s = time.time() - t0
    srv = Server(0, loaders=loaders, copy_engine_uploads=copy_engine_uploads, large_blocks_per_sm=large_bps,
                 large_layout_blocks_per_sm=large_layout_bps,
                 max_large_loads=None if max_large_loads < 0 else max_large_loads,
                 small_sms=None if small_sms < 0 else small_sms,
                 small_aging_us=None if small_aging_us < 0 else small_aging_us)
    try:
        for s in sorted(pool):
            g, c = pool[s][0]
            info = srv.wait(srv.submit_csr(g, c))
            assert want is None or info.count == want[(s, 0)]
        runs = [serve_once(srv, pool, max_scale, r, duration, seed=7 + k, want=want, trace=trace)
                for k, r in enumerate(rates)]
        st = srv.stats()
    finally:
        srv.close()
    del keep
    return {"runs": runs, "pool_graphs": sum(len(v) for v in pool.values()), "generate_s": round(gen_s, 1),
            "oracle_s": round(oracle_s, 1), "launches": st.launches, "max_batch": st.max_batch,
            "loaders": loaders, "pinned_requests": pin, "large_blocks_per_sm": large_bps or 3,
            "large_layout_blocks_per_sm": large_layout_bps or 2, "small_sms": small_sms,
            "small_aging_us": small_aging_us,
            "small_uploads": "copy engines" if copy_engine_uploads or not pin else "kernel reads",
            "workload": f"serving: Poisson arrivals, R-MAT scale 12+Geom(0.3) <= {max_scale}, ef 16"}


def run_serve(args):
    rates = [float(x) for x in args.rates.split(",")] if args.rates else [args.rate]
    trace = [] if args.trace else None
    sv = measure_serve(args.serve_max_scale, rates, args.duration, args.loaders, bool(args.pin),
                       args.copy_engine_uploads, check=not args.no_check, trace=trace, large_bps=args.large_bps,
                       large_layout_bps=args.large_layout_bps, max_large_loads=args.max_large_loads,
                       small_sms=args.small_sms, small_aging_us=args.small_aging_us)
    if args.trace:
        with open(args.trace, "w") as f:
            json.dump({"fields": ["scale", "m", "submit_ns", "load_ns", "ready_ns", "launch_ns", "done_ns", "batch"],
                       "requests": trace}, f)
    peak = max(r["value"] for r in sv["runs"])
    for r in sv["runs"]:
        res = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": r["requests"],
               "warmup": sv["pool_graphs"], "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "u32", "data": "synthetic",
               "config": {"workload": f"{sv['workload']}, {r['rate']:g} req/s for {r['duration_s']:g} s",
                          **{k: v for k, v in sv.items() if k not in ("runs", "workload")}},
               **{k: v for k, v in r.items() if k not in ("value", "unit")},
               "frac_of_sweep_peak": r["value"] / peak}
        print(json.dumps(res), flush=True)


def child_line(extra) -> dict | None:
    """Run this script with `extra` arguments in a child process and return
    its last JSON line (None, with the error, if it failed)."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__), *extra], capture_output=True, text=True,
                       timeout=1200)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"exit {r.returncode}: {r.stderr.strip()[-400:]}"}
    return json.loads(lines[-1])


def main():
    args = parse()
    if args.config == "batch":
        return run_batch(args)
    if args.config == "serve":
        return run_serve(args)
    if args.config == "hybrid":
        return run_hybrid(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local)  # before the NCCL communicator exists
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        res = run_reference(args, rank)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    from bbtc_b200 import Context, Graph, graphs, options

    torch.cuda.set_device(local)
    ctx = Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    g, cuts, gen_s = make_graph(args, args.seed + rank)
    balg = g.algorithmic_bytes()
    st = Graph.from_csr(ctx, g, cuts)
    layout_ms = st.info().layout_ms
    device_bytes = st.info().device_bytes
    o = options(mode="persistent", kernel=args.kernel, bitmap_words=args.bitmap_words, unit_work=args.unit_work,
                cuda_graph=True, occupancy=args.occupancy, warps_per_block=args.warps)
    tuned = None
    if not args.no_autotune and not args.bitmap_words and not args.occupancy and args.kernel in ("auto", "fused"):
        # the library's sweep (every point must give the same count) over the
        # fused kernel's shared buffer and register budget, outside the timed
        # region and uncached, so every run tunes for the GPU it runs on
        from bbtc_b200 import autotune
        t0 = time.perf_counter()
        o, tune_ms = autotune.sweep(st, base=o, bitmap_words=(768, 1024, 1536), occupancy=(4, 5, 6),
                                    warps_per_block=(8,), unit_work=(0, 512), repeats=5)
        o.use_cuda_graph = 1
        tuned = {f: getattr(o, f) for f in ("bitmap_words", "warps_per_block", "unit_work", "occupancy")}
        tuned.update(sweep_ms=round(tune_ms, 3), sweep_s=round(time.perf_counter() - t0, 2),
                     space="bitmap_words 768/1024/1536 x occupancy 4/5/6 x units automatic / 512 probes, "
                           "8 warps")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def timed_counts(opts, steps, warmup):
        for _ in range(warmup):
            st.count(opts=opts)
        times, counts = [], set()
        launches = 0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)  # evicts L2 (126 MB) between timed steps
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st.count_async(opts=opts)
                e1.record(stream)
            counts.add(st.count_wait())
            launches += st.last_launches()
            times.append(e0.elapsed_time(e1))
        return times, counts, launches

    # --- persistent form (the headline value) ---
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    times, counts, launches = timed_counts(o, args.steps, args.warmup)
    clk = clocks.stop()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t_mean = sum(times) / len(times) / 1e3
    assert len(counts) == 1, f"count changed between steps: {counts}"
    count = counts.pop()
    t_max = t_mean
    m_total = g.m
    if dist is not None:
        # the only exchange: edges and counts summed, the slowest rank's time
        from bbtc_b200 import multi
        m_total, count_total, t_max = multi.aggregate(dist, g.m, count, t_mean, device=f"cuda:{local}")
    value = m_total / t_max

    # --- plain form (one launch per task) ---
    plain = None
    if not args.no_plain:
        po = options(mode="plain", kernel=args.kernel, bitmap_words=args.bitmap_words, unit_work=args.unit_work,
                     cuda_graph=False)
        ptimes, pcounts, plaunches = timed_counts(po, max(3, args.steps // 2), 2)
        assert pcounts == {count}, f"plain form disagrees: {pcounts} vs {count}"
        pt = sum(ptimes) / len(ptimes) / 1e3
        plain = {"value": g.m / pt, "unit": UNIT, "ms_per_step": pt * 1e3,
                 "launches_per_step": plaunches // len(ptimes), "persistent_over_plain": pt / t_mean}
        # the same per-task kernel as the plain form, every task's units in one
        # persistent launch from the device queue: separates the queue's gain
        # from the fused task rows' algorithmic gain
        qo = options(mode="persistent", kernel="bitmap", bitmap_words=args.bitmap_words, cuda_graph=True)
        tl = st.task_list(sorted=True)
        qtimes, qcounts = [], set()
        for i in range(2 + max(3, args.steps // 2)):
            with torch.cuda.stream(stream):
                flush.fill_(1)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st.count_async(tl, opts=qo)  # an explicit per-task kernel: the task queue, not task rows
                e1.record(stream)
            qcounts.add(st.count_wait())
            if i >= 2:
                qtimes.append(e0.elapsed_time(e1))
        assert qcounts == {count}, f"per-task queue disagrees: {qcounts} vs {count}"
        qt = sum(qtimes) / len(qtimes) / 1e3
        plain["persistent_per_task"] = {
            "value": g.m / qt, "unit": UNIT, "ms_per_step": qt * 1e3, "launches_per_step": 1,
            "kernel": "per-task bitmap (k_count_queue), every task of the sorted list in one launch",
            "over_plain": pt / qt, "fused_over_per_task": qt / t_mean}

    # --- e2e through the C ABI from pinned host buffers ---
    e2e = None
    if not args.no_e2e:
        ip = torch.from_numpy(g.indptr.view(np.int32)).pin_memory()
        ix = torch.from_numpy(g.indices.view(np.int32)).pin_memory()
        from bbtc_b200 import core
        # a new graph every step: no CUDA graph capture (it would be replayed once)
        oe = options(mode="persistent", kernel=args.kernel, bitmap_words=o.bitmap_words, unit_work=o.unit_work,
                     cuda_graph=False, occupancy=o.occupancy, warps_per_block=o.warps_per_block)
        e2e_t, warm_layout = [], []
        for i in range(args.warmup + max(3, args.steps // 2)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            h = core.Graph.upload_ptrs(ctx, g.n, ip.data_ptr(), ix.data_ptr(), g.m, cuts)
            c2 = h.count(opts=oe)
            lm = h.info().layout_ms
            h.free()
            t1 = time.perf_counter()
            assert c2 == count
            if i >= args.warmup:
                e2e_t.append(t1 - t0)
                warm_layout.append(lm)
        te = statistics.median(e2e_t)
        e2e = {"value": g.m / te, "unit": UNIT, "ms_per_step": te * 1e3,
               "h2d_bytes_per_step": int(4 * (g.n + 1) + 4 * g.m + 4 * len(cuts)),
               "d2h_bytes_per_step": 8, "layout_ms": statistics.median(warm_layout),
               "note": "upload (H2D from pinned memory) + device layout build + persistent count + 8-byte "
                       "readback, wall clock; the library's control copies (tile statistics, task queue, "
                       "< 1 MB) are not in the byte counts"}

    # --- CPU baseline: the reference's own CPU path on this host ---
    cpu = None
    ref_match = None
    if not args.no_cpu and rank == 0 and world == 1:
        import oracle
        if oracle.ref_available():
            threads = args.cpu_threads or os.cpu_count()
            part = "pal" if args.partitioner.startswith("pal") else args.partitioner
            rcuts = oracle.ref_cuts(g.n, g.indptr, g.indices, args.ncut, part)
            rc, secs = oracle.ref_count(g.n, g.indptr, g.indices, rcuts, nthreads=threads, repeat=1)
            ref_match = (rc == count)
            cpu = {"value": g.m / secs[0], "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": "the full workload once: the reference's NoOfTriangles() over all tasks of the "
                             "same graph, cut by the reference's own SARMA partitioner (oracle/_ref, built from "
                             "the reference's sources)",
                   "seconds": secs[0], "count_matches_gpu": ref_match}

    # --- the reference's own GPU executable (its one-launch-per-task form), same graph ---
    ref_gpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        import oracle
        if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "bbtc_gpu")):
            try:
                part = "pal" if args.partitioner.startswith("pal") else args.partitioner
                r = oracle.ref_gpu_cli(g.n, g.indptr, g.indices, part, args.ncut, repeat=3, timeout=900)
                tr = statistics.median(r["count_seconds"])
                ref_gpu = {"value": g.m / tr, "unit": UNIT, "ms_per_step": tr * 1e3, "triangles": r["triangles"],
                           "count_matches_gpu": r["triangles"] == count, "copy_s": r["copy_seconds"],
                           "layout_s": r["layout_seconds"], "over_reference_gpu": tr / t_mean,
                           "run": "oracle/_ref/bbtc_gpu (the reference's src/bbtc.cu built unmodified for "
                                  "sm_100a) --ngpu 1 --border -1 --copy-first --repeat 3, its own SARMA cuts; "
                                  "median 'Triangle Counting Execution Time'"}
            except Exception as e:  # the baseline is reported, not required
                ref_gpu = {"error": str(e)[-300:]}

    # --- hybrid GPU + CPU execution (bb_tc.cpp:142-252) on the same graph, in a
    # child process (its CPU worker threads and their memory stay out of this one) ---
    hybrid = None
    if rank == 0 and world == 1 and not args.no_hybrid:
        hybrid = child_line(["--config", "hybrid", "--family", args.family, "--scale", str(args.scale),
                             "--edge-factor", str(args.edge_factor), "--seed", str(args.seed), "--ncut",
                             str(args.ncut), "--partitioner", args.partitioner, "--steps", "3", "--warmup", "1"])
        if hybrid is not None and "error" not in hybrid:
            hybrid["count_matches"] = hybrid.get("config", {}).get("triangles") == count

    # --- batched launch and serving sub-records (576 graphs in one launch; Poisson request streams; short) ---
    # each in a fresh child process, as a deployment runs them (host threads and
    # device memory pools of this process do not carry over)
    batch_rec = serve_rec = None
    if rank == 0 and world == 1 and not args.no_batch:
        batch_rec = child_line(["--config", "batch", "--batch-max-scale", str(args.sub_batch_max_scale),
                                "--steps", "5", "--warmup", "2", "--batch-plain-steps", "0"])
    if rank == 0 and world == 1 and not args.no_serve:
        rate = args.sub_serve_rate or (0.8 * SERVE_PEAK_RPS)
        serve_rec = child_line(["--config", "serve", "--rate", f"{rate:g}", "--duration",
                                f"{args.sub_serve_duration:g}", "--serve-max-scale", "22"])
        if serve_rec is not None:
            serve_rec.update({"peak_rps": SERVE_PEAK_RPS, "rate_over_peak": rate / SERVE_PEAK_RPS,
                              "peak_note": "SERVE_PEAK_RPS: the request rate where edges/s stopped growing in "
                                           "`bench.py --config serve --rates ...` (profiles/serving_sweep.md)"})

    peak, peak_kind = peaks()
    fb = g.fused_bytes(cuts) if args.kernel in ("auto", "fused") else None
    model_bytes = fb["bytes"] if fb else balg
    achieved = model_bytes / t_mean / 1e9
    traffic, traffic_note = load_traffic(args.family, args.scale, args.ncut)
    res = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"{workload_name(args)} {args.partitioner} "
                               f"ncut {args.ncut}", "n": g.n, "m": g.m, "P": args.ncut,
                   "partitioner": args.partitioner, "mode": "persistent (one launch, device queue, CUDA graph)",
                   "kernel": args.kernel, "triangles": count if world == 1 else count_total,
                   "layout_ms_first": layout_ms,
                   "layout_ms": e2e["layout_ms"] if e2e else layout_ms, "device_bytes": device_bytes, "generate_s": round(gen_s, 2),
                   "l2": "block CSR larger than L2, plus a 256 MiB fill between timed steps (excluded)",
                   "launch": {f: (getattr(o, f) or "auto") for f in ("bitmap_words", "warps_per_block", "unit_work",
                                                                       "occupancy")}, "autotuned": tuned,
                   "parallelism": "replicas per GPU" if world > 1 else "single GPU"},
        "plain": plain,
        "e2e": e2e,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "model_bytes": model_bytes, "model": ("fused task rows" if fb else "B_alg"),
                     "model_parts": fb,
                     "peak_note": "of measured (MEASURED_PEAKS.json hbm_gbs)"
                     if peak_kind == "measured" else "of fallback",
                     "algorithmic_bytes_merge": balg, "merge_frac": balg / t_mean / 1e9 / peak,
                     "dram_gbs": (traffic / t_mean / 1e9) if traffic else None,
                     "dram_frac": (traffic / t_mean / 1e9 / peak) if traffic else None,
                     "note": ("achieved = model bytes / count time (CUDA events on the library's stream). Model "
                              "(fused task rows, the default path): 8 B per streamed (32-id word, bit mask) pair "
                              "(in-edge (u, v) streams N+(u) from v's word to the row's end), 8 B per in-edge "
                              "record, and per pivot visit its word pairs plus 28 B of row pointers and bounds -- "
                              "each byte once per use, no cache reuse. merge_frac: the same time against B_alg = "
                              "4m + 4 sum over edges of d+(u) + d+(v), the ids a merge intersection streams, "
                              "which this kernel does not read. dram_gbs: ncu DRAM traffic of one launch over the "
                              "same time" + (f"; traffic: {traffic_note}" if traffic_note else ""))},
        "cpu_baseline": cpu,
        "reference_gpu": ref_gpu,
        "hybrid": hybrid,
        "batch": batch_rec,
        "serve": serve_rec,
        "gpu_launches": launches,
        "clocks": clk,
        "triangles_per_sec": (count / t_mean) if world == 1 else None,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)
    st.free()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

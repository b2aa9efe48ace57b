"""Host logic for several GPUs (one process per GPU, torch.distributed).

The reference stripes tasks over GPUs by worker index (src/triangle_counting/
bb_tc.cpp:144-146) and sums one u64 counter per GPU stream on the host
(bb_tc.cpp:242-249).  Tasks are independent, so the only exchange is that sum.

* :func:`aggregate` -- after a timed region: total edges and triangles (sum)
  and the slowest rank's time (max), one all_reduce each.
* :func:`shard_tasks` -- a cost-balanced split of one graph's task list over
  ranks (longest-processing-time greedy), for counting one graph on several
  GPUs; each rank counts its share with ``Graph.count(tasks=...)``.
"""
from __future__ import annotations

import heapq

import numpy as np


def aggregate(dist, m: int, count: int, seconds: float, device="cpu") -> tuple[int, int, float]:
    import torch
    mc = torch.tensor([m, count], dtype=torch.int64, device=device)
    dist.all_reduce(mc, op=dist.ReduceOp.SUM)
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return int(mc[0].item()), int(mc[1].item()), float(t.item())


def shard_tasks(costs, world: int) -> list[np.ndarray]:
    """Indices of the tasks each rank runs: heaviest first onto the least
    loaded rank.  Every task lands on exactly one rank."""
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    shards: list[list[int]] = [[] for _ in range(world)]
    for t in order:
        load, r = heapq.heappop(heap)
        shards[r].append(int(t))
        heapq.heappush(heap, (load + float(costs[t]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def task_costs(nnz: np.ndarray, tile_deg: np.ndarray, tasks: np.ndarray) -> np.ndarray:
    """The reference's task weight nnz(ab) * max(tile_deg(bc), tile_deg(ac))
    (include/utils/tasks.hpp:21-23), NaN (empty parts) as 0."""
    w = nnz[tasks["ab"]].astype(np.float64) * np.maximum(tile_deg[tasks["bc"]], tile_deg[tasks["ac"]])
    return np.nan_to_num(w, nan=0.0)

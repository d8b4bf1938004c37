"""Sharding of a batch of independent systems over ranks.

The reference is single-process (README.md:327); its only parallelism is
shared-memory threading.  A batch of independent structures (the training set
of design_matrix, ACE/fitting.jl:18-67) shards without any data exchange:
every rank evaluates its own systems with one batched launch, and the
per-system results are gathered once at the end.

  system_costs   expected directed edges per system, n·(n/V)·(4/3)π c³
  shard          greedy longest-processing-time bin packing of the costs
  gather_rows    all_gather of per-system result rows (padded to the largest
                 shard) back into the original system order, on any
                 torch.distributed backend (NCCL on GPUs, gloo on CPUs)
"""
from __future__ import annotations

import heapq
import math

import numpy as np


def system_costs(systems, cutoff):
    """Expected directed neighbour count of each system (uniform density)."""
    ball = 4.0 / 3.0 * math.pi * cutoff ** 3
    out = np.zeros(len(systems))
    for k, s in enumerate(systems):
        n = len(s.species)
        V = abs(float(np.linalg.det(np.asarray(s.H, np.float64).reshape(3, 3))))
        out[k] = n * (n / V) * ball if V > 0 else n * n
    return out


def shard(costs, world):
    """Greedy LPT: systems in decreasing cost (ties by index) go to the least
    loaded rank (ties by rank).  Returns one sorted index list per rank."""
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        parts[r].append(k)
        heapq.heappush(heap, (load + float(costs[k]), r))
    return [sorted(p) for p in parts]


def gather_rows(local_rows, parts, rank, group=None, device=None):
    """local_rows [len(parts[rank]), k] float64 → [nsys, k] on every rank."""
    import torch
    import torch.distributed as dist
    world = len(parts)
    k = local_rows.shape[1] if local_rows.ndim == 2 else 1
    width = max(len(p) for p in parts)
    buf = torch.zeros((width, k), dtype=torch.float64, device=device)
    if len(parts[rank]):
        buf[: len(parts[rank])] = torch.as_tensor(np.asarray(local_rows).reshape(len(parts[rank]), k), device=device)
    bufs = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(bufs, buf, group=group)
    nsys = sum(len(p) for p in parts)
    out = np.zeros((nsys, k))
    for r in range(world):
        rows = bufs[r].cpu().numpy()
        for i, s in enumerate(parts[r]):
            out[s] = rows[i]
    return out

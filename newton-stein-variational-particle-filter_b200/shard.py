"""Filters across GPUs: one process per GPU, no per-tick exchange.

Filters are independent, so a tick never needs data from another GPU: each
rank steps its own share of the filters with one persistent launch per tick.
Shares are balanced by the cost of a tick, N^2 times the Stein-iteration
bound, with a largest-first greedy assignment.  At the end of a run the
per-filter FP64 log-likelihood sums are gathered with one all_gather (NCCL on
GPUs, gloo on CPU); run time is the maximum over ranks.
"""
from __future__ import annotations

import heapq

import numpy as np


def tick_cost(ns, max_steps) -> np.ndarray:
    ns = np.asarray(ns, dtype=np.float64)
    steps = np.broadcast_to(np.asarray(max_steps, dtype=np.float64), ns.shape)
    return ns * ns * np.maximum(steps, 1.0)


def partition(ns, max_steps, world: int) -> list[np.ndarray]:
    """Filter indices of every rank, balanced by tick cost (largest first to
    the least-loaded rank).  Each rank's indices are returned sorted."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cost = tick_cost(ns, max_steps)
    order = np.argsort(-cost, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shares = [[] for _ in range(world)]
    for f in order:
        load, r = heapq.heappop(heap)
        shares[r].append(int(f))
        heapq.heappush(heap, (load + float(cost[f]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shares]


def imbalance(ns, max_steps, shares) -> float:
    """max rank load / mean rank load."""
    cost = tick_cost(ns, max_steps)
    loads = np.array([cost[s].sum() for s in shares])
    return float(loads.max() / max(loads.mean(), 1e-30))


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar over the default process group."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_by_filter(local_idx, local_values, n_filters: int, device=None) -> np.ndarray:
    """Every rank contributes the values of its filters; every rank receives
    the full [n_filters] array in global filter order (one all_gather)."""
    import torch
    import torch.distributed as dist

    local_idx = np.asarray(local_idx, dtype=np.int64)
    local_values = np.asarray(local_values, dtype=np.float64)
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        out = np.full(n_filters, np.nan)
        out[local_idx] = local_values
        return out
    world = dist.get_world_size()
    # pad every share to the longest so all ranks send equal-sized tensors
    sizes = torch.tensor([local_idx.shape[0]], dtype=torch.int64, device=device)
    all_sizes = [torch.zeros_like(sizes) for _ in range(world)]
    dist.all_gather(all_sizes, sizes)
    m = int(max(int(s.item()) for s in all_sizes))
    buf = torch.full((m, 2), -1.0, dtype=torch.float64, device=device)
    buf[: local_idx.shape[0], 0] = torch.from_numpy(local_idx.astype(np.float64))
    buf[: local_idx.shape[0], 1] = torch.from_numpy(local_values)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.full(n_filters, np.nan)
    for p in parts:
        a = p.cpu().numpy()
        valid = a[:, 0] >= 0
        out[a[valid, 0].astype(np.int64)] = a[valid, 1]
    return out

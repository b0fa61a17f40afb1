"""Spreading independent systems over GPUs (one process per GPU).

The systems of a batch are independent, so ranks exchange nothing while they
solve: each rank takes a share of the systems, solves it with its own
``BatchedSolver`` and the per-system records are gathered at the end.  Shares
are balanced by nonzeros with longest-processing-time bins (largest system
first, always onto the least-loaded rank).  Timing across ranks is the
maximum of the per-rank device times.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition_by_nnz(nnz, world: int):
    """Index arrays (ascending) of the systems each rank solves."""
    nnz = np.asarray(nnz, np.int64)
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    owner = np.empty(nnz.shape[0], np.int64)
    for s in np.argsort(-nnz, kind="stable"):
        load, r = heapq.heappop(heap)
        owner[s] = r
        heapq.heappush(heap, (load + int(nnz[s]), r))
    return [np.nonzero(owner == r)[0] for r in range(world)]


def local_rows(row_off, systems):
    """Row offsets of the rank's own block-diagonal stack of `systems`."""
    row_off = np.asarray(row_off, np.int64)
    idx = np.asarray(systems, np.int64)
    sizes = row_off[idx + 1] - row_off[idx]
    loc = np.zeros(idx.shape[0] + 1, np.int64)
    loc[1:] = np.cumsum(sizes)
    return loc


def gather_records(values, systems, n_systems: int, group=None, device=None):
    """All ranks' per-system values (one per local system) merged into one
    array indexed by global system id, on every rank.  device: where the
    exchanged tensors live (a CUDA device for the NCCL backend, None = CPU
    for gloo)."""
    import torch
    import torch.distributed as dist

    values = np.asarray(values, np.float64)
    systems = np.asarray(systems, np.int64)
    world = dist.get_world_size(group)
    cnt = torch.tensor([systems.shape[0]], dtype=torch.int64, device=device)
    counts = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(counts, cnt, group=group)
    m = max(1, int(max(c.item() for c in counts)))
    pad_i = torch.full((m,), -1, dtype=torch.int64)
    pad_v = torch.zeros(m, dtype=torch.float64)
    pad_i[: systems.shape[0]] = torch.from_numpy(systems)
    pad_v[: systems.shape[0]] = torch.from_numpy(values)
    pad_i, pad_v = pad_i.to(device), pad_v.to(device)
    all_i = [torch.empty(m, dtype=torch.int64, device=device) for _ in range(world)]
    all_v = [torch.empty(m, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(all_i, pad_i, group=group)
    dist.all_gather(all_v, pad_v, group=group)
    out = np.full(n_systems, np.nan)
    for i, v in zip(all_i, all_v):
        i, v = i.cpu(), v.cpu()
        keep = i >= 0
        out[i[keep].numpy()] = v[keep].numpy()
    return out


def max_over_ranks(value: float, group=None, device=None) -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())

"""Source sharding for one process per GPU.

Every step of the point-source path is independent per source once the small
shared tables (effective area, King grids, livetime efficiency, map geometry)
are replicated, so N GPUs run N independent pipelines on disjoint sets of
sources and exchange nothing on the data path.  The reference runs all sources
in one process (its source loops are OpenMP, schedule(static, 16):
model_map/mm_cubature/cubature.implementation.cxx:39).

``shard_sources`` assigns sources to ranks by longest-processing-time greedy
over an estimated cost (pixels x energies by default, so uneven cutouts
balance); ``gather_rows`` is the one optional collective, an all-gather of small
per-source results (map totals, 1/integral, correction factors) back into
global source order.
"""
from __future__ import annotations

import heapq
from typing import Optional, Sequence

import numpy as np


def shard_sources(n_sources: int, world: int, cost: Optional[Sequence[float]] = None) -> list:
    """Split sources 0..n-1 over ``world`` ranks.  Returns one sorted index array
    per rank.  With equal costs the shards are contiguous blocks whose sizes
    differ by at most one; otherwise the heaviest source goes to the least
    loaded rank first (ties to the lower rank)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    if cost is None:
        bounds = [n_sources * r // world for r in range(world + 1)]
        return [np.arange(bounds[r], bounds[r + 1]) for r in range(world)]
    cost = np.asarray(cost, dtype=np.float64)
    if cost.shape != (n_sources,):
        raise ValueError("cost needs one entry per source")
    heap = [(0.0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for s in sorted(range(n_sources), key=lambda i: (-cost[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(s)
        heapq.heappush(heap, (load + cost[s], r))
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def gather_rows(local: np.ndarray, index: np.ndarray, n_sources: int, group=None) -> np.ndarray:
    """All-gather per-source rows (``local[i]`` belongs to global source
    ``index[i]``) into an array in global source order, over torch.distributed
    (CUDA tensors with NCCL, CPU tensors with gloo).  Every rank calls it once
    with its own shard, in the same order as the other collectives."""
    import torch
    import torch.distributed as dist

    local = np.ascontiguousarray(local, dtype=np.float64)
    world = dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" \
        else torch.device("cpu")
    width = int(np.prod(local.shape[1:])) if local.ndim > 1 else 1
    n = torch.tensor([len(index)], dtype=torch.int64, device=dev)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    buf = torch.zeros((max(counts), 1 + width), dtype=torch.float64, device=dev)
    buf[: len(index), 0] = torch.as_tensor(np.asarray(index, dtype=np.float64), device=dev)
    buf[: len(index), 1:] = torch.as_tensor(local.reshape(len(index), width), device=dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = np.zeros((n_sources, width), dtype=np.float64)
    for r in range(world):
        p = parts[r][: counts[r]].cpu().numpy()
        out[p[:, 0].astype(np.int64)] = p[:, 1:]
    return out.reshape((n_sources,) + local.shape[1:])

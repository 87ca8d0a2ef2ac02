"""Multi-GPU work partitioning for the cloud march.

The forward march has no exchange step: every primary ray is independent, so
views, frames and rows shard across ranks with no data-path collective.  One
process per GPU; read-only inputs (noise, LUTs, weather) are replicated on
each device by the host.

* `partition_views`  — largest-first assignment of whole views/frames to ranks
  by an estimated cost (pixels x primary steps x layers), the LPT schedule.
* `row_bands`        — split one large view into contiguous row bands with
  equal estimated cost (rows above the horizon cost more than ground rows).
* `gather_rows`      — all-gather of the bands back into one image, for when a
  single composited frame is required on every rank (uses the process
  group's backend: NCCL over NVLink on GPUs, gloo on CPU).
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Band:
    rank: int
    y0: int
    y1: int


def view_cost(width: int, height: int, steps: int, layers: int) -> float:
    return float(width) * float(height) * float(max(steps, 1)) * float(max(layers, 1))


def partition_views(costs, world_size: int) -> list[list[int]]:
    """Assign items (indices into `costs`) to `world_size` ranks, largest cost
    first onto the currently lightest rank.  Deterministic (ties by index)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world_size)]
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(v) for v in out]


def row_bands(height: int, world_size: int, row_weights=None) -> list[Band]:
    """Contiguous row bands, one per rank, balancing the sum of `row_weights`
    (uniform when None).  Every row belongs to exactly one band."""
    if world_size < 1 or height < 1:
        raise ValueError("need height >= 1 and world_size >= 1")
    w = np.ones(height) if row_weights is None else np.asarray(row_weights, np.float64)
    if w.shape != (height,) or np.any(w < 0):
        raise ValueError("row_weights must be a non-negative vector of length height")
    if w.sum() <= 0:
        w = np.ones(height)
    cum = np.concatenate([[0.0], np.cumsum(w)])
    cuts = [0]
    for r in range(1, world_size):
        target = cum[-1] * r / world_size
        y = int(np.searchsorted(cum, target, side="left"))
        cuts.append(min(max(y, cuts[-1]), height))
    cuts.append(height)
    return [Band(r, cuts[r], cuts[r + 1]) for r in range(world_size)]


def gather_rows(local, band: Band, bands: list[Band], group=None):
    """All-gather row bands (tensors of shape (rows, W, C)) into the full
    image on every rank.  Bands may differ in height, so each is padded to
    the largest band for the collective and trimmed afterwards."""
    import torch
    import torch.distributed as dist
    hmax = max(b.y1 - b.y0 for b in bands)
    pad = torch.zeros((hmax,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[: band.y1 - band.y0] = local
    parts = [torch.empty_like(pad) for _ in bands]
    dist.all_gather(parts, pad, group=group)
    return torch.cat([p[: b.y1 - b.y0] for p, b in zip(parts, bands)], dim=0)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """Max of a scalar (e.g. a device-timed step) over all ranks."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def allreduce_gradient(grad, acc, group=None):
    """The adjoint's exchange step: pixels are sharded by row bands, so each
    rank holds a partial d loss / d grid (and its share of the loss and of
    d loss / d density_scale in `acc`); one sum all-reduce of each gives
    every rank the whole image's values.  In place; a no-op on one rank."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=group)
    return grad, acc

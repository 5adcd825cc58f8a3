"""Sharding of the workloads that partition across GPUs: one process per GPU, no collective on the data path.

* Ensembles: independent systems are split over the ranks by their work (n_step x bodies x (bodies + 8):
  the two O(n^2) pair sweeps and the per-body update of every stage). Every rank computes the same split
  from the same inputs, so no communication is needed to agree on it. The reference balances work items
  over threads with a randomised search of swaps between subsets (src/math/distribute.h:18-100); here the
  split is deterministic: longest processing time first, then moves and swaps between the most and the
  least loaded rank while they lower the largest load.
* Massless particles: one particle set is cut into contiguous index ranges, one per rank; the perturbers are
  replicated and integrated by every rank (they are few). The only collective is one gather of the final
  states to rank 0.
"""
from __future__ import annotations

import numpy as np


def member_cost(n_bodies: int, n_step: int) -> float:
    """Work estimate of integrating one system: n_step x n (n + 8)."""
    return float(abs(n_step)) * n_bodies * (n_bodies + 8)


def partition(costs, world: int) -> list[list[int]]:
    """Split items of the given costs into `world` lists of indices with loads as equal as possible
    (deterministic: ties broken by index). Every index appears in exactly one list, in ascending order."""
    costs = np.asarray(costs, dtype=float)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    parts: list[list[int]] = [[] for _ in range(world)]
    load = np.zeros(world)
    for i in order:
        r = int(np.argmin(load))          # the first least-loaded rank
        parts[r].append(i)
        load[r] += costs[i]
    # refinement: move or swap one item between the heaviest and the lightest rank while that lowers the
    # heavier of the two (and so never raises the largest load)
    for _ in range(4 * len(costs)):
        hi, lo = int(np.argmax(load)), int(np.argmin(load))
        gap = load[hi] - load[lo]
        best, best_gain = None, 0.0
        for a in parts[hi]:
            # moving a (d = its cost) or swapping it with b (d = cost difference) leaves the two ranks at
            # hi - d and lo + d: it helps when 0 < d < gap, by min(d, gap - d)
            for b in [None] + parts[lo]:
                d = costs[a] - (0.0 if b is None else costs[b])
                if 0 < d < gap and min(d, gap - d) > best_gain:
                    best, best_gain = (a, b), min(d, gap - d)
        if best is None or best_gain <= 1e-12 * max(1.0, gap):
            break
        a, b = best
        parts[hi].remove(a)
        parts[lo].append(a)
        load[hi] -= costs[a]
        load[lo] += costs[a]
        if b is not None:
            parts[lo].remove(b)
            parts[hi].append(b)
            load[lo] -= costs[b]
            load[hi] += costs[b]
    return [sorted(p) for p in parts]


def particle_slice(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous index range [lo, hi) of `rank`'s particles out of n (sizes differ by at most one)."""
    lo = n * rank // world
    return lo, n * (rank + 1) // world


def gather_rows(local: np.ndarray, n_total: int, pg=None, device=None):
    """Gather every rank's [rows][n_r] slice (rank order = particle order) into rank 0's [rows][n_total] array;
    other ranks get None. One all-gather of padded slices over the process group (NCCL on GPUs, gloo on CPUs)."""
    import torch
    import torch.distributed as dist
    if pg is None:
        return local
    world, rank = dist.get_world_size(pg), dist.get_rank(pg)
    width = max(particle_slice(n_total, world, r)[1] - particle_slice(n_total, world, r)[0] for r in range(world))
    pad = np.zeros((local.shape[0], width), dtype=local.dtype)
    pad[:, :local.shape[1]] = local
    t = torch.from_numpy(pad)
    if device is not None:
        t = t.to(device)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=pg)
    if rank != 0:
        return None
    cols = []
    for r, o in enumerate(outs):
        lo, hi = particle_slice(n_total, world, r)
        cols.append(o.cpu().numpy()[:, :hi - lo])
    return np.concatenate(cols, axis=1)

"""Multi-GPU layout of the CLE: one process per GPU, cells sharded by global index.

Cells of a network without population dynamics are independent and every random
increment is keyed by the global cell index, so a shard run with
`cell_offset = first global cell` reproduces exactly the rows of a single-GPU
run.  No collective is needed on the data path.  Networks with a Moran
population couple their cells at division and are placed whole on one rank
(`shard_networks`).  The only collective is the FP64 reduction of per-gene
moment sums (`moment_sums` + `allreduce_moments`), a few KB per call.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np


def shard_cells(n_cells: int, world: int, rank: int) -> Tuple[int, int]:
    """(offset, count) of this rank's contiguous slice; sizes differ by at most one."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank / world size")
    base, extra = divmod(int(n_cells), world)
    count = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    return offset, count


def shard_networks(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy longest-processing-time placement of whole networks on ranks."""
    order = sorted(range(len(costs)), key=lambda i: -costs[i])
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: load[k])
        out[r].append(i)
        load[r] += costs[i]
    for lst in out:
        lst.sort()
    return out


def shard_network_ranges(costs: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Contiguous ranges [lo, hi) of networks, one per rank (empty ones at the end), whose
    largest total cost is the smallest a contiguous split allows (bisection on that bound,
    each range filled greedily).  Contiguous ranges keep each network's batch index offset
    by the range start, so a batch call per range with base stream `stream + lo` gives every
    network the Philox stream it has in one call over all of them."""
    if world <= 0:
        raise ValueError("bad world size")
    c = [float(x) for x in costs]
    if any(x < 0 for x in c):
        raise ValueError("costs must be non-negative")
    n = len(c)

    def n_ranges(bound):
        k, s = 1, 0.0
        for x in c:
            if s + x > bound:
                k, s = k + 1, x
            else:
                s += x
        return k

    lo, hi = max(c, default=0.0), sum(c)
    for _ in range(200):
        if hi - lo <= 1e-12 * max(hi, 1.0):
            break
        mid = 0.5 * (lo + hi)
        if n_ranges(mid) <= world:
            hi = mid
        else:
            lo = mid
    ranges, start, s = [], 0, 0.0
    for i, x in enumerate(c):
        if s + x > hi and i > start:
            ranges.append((start, i))
            start, s = i, 0.0
        s += x
    ranges.append((start, n))
    while len(ranges) < world:
        ranges.append((n, n))
    return ranges


def moment_sums(X: np.ndarray) -> np.ndarray:
    """Per-column [count, sum, sum of squares] in FP64 for a cells x genes matrix."""
    Xd = np.asarray(X, dtype=np.float64)
    return np.stack([np.full(Xd.shape[1], Xd.shape[0], dtype=np.float64), Xd.sum(0), (Xd * Xd).sum(0)])


def allreduce_moments(sums: np.ndarray, group=None) -> np.ndarray:
    """Sum the per-rank moment sums over the process group (NCCL on GPUs, gloo on CPU)."""
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.as_tensor(np.ascontiguousarray(sums), dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def moments_from_sums(sums: np.ndarray):
    """(mean, unbiased variance) per column from [count, sum, sum of squares]."""
    n, s, ss = sums
    mean = s / n
    var = (ss - n * mean * mean) / np.maximum(n - 1, 1)
    return mean, var

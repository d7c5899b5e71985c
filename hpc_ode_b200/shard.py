"""Cell sharding over several GPUs of one node: one process per GPU, cells
split into contiguous ranges, no collective on the data path.

Cells are independent (each runs its own BDF), so a batch splits into one
contiguous range per rank.  Ranges are balanced by a per-cell cost: by default
a proxy from the initial temperature (cells near ignition take many more BDF
steps than frozen or fully burnt ones); a flow solver that calls every time
step can pass the step counts of its previous call instead.  Each rank
integrates its range on its own GPU; the only communication is the optional
gather of results to one rank (``gather_to``), which is plumbing, not part of
the integration.

The reference has no multi-GPU path; its GPU integrator splits a mesh into
memory-sized batches on one device (CVodeIntegratorGPU::integrate,
src/Integrators/CVodeIntegratorGPU.cpp:30-42).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def temperature_cost(T: np.ndarray) -> np.ndarray:
    """Relative cost proxy per cell from the initial temperature: frozen cells
    (below ~900 K) take a few steps, cells in the ignition window the most."""
    T = np.asarray(T, dtype=np.float64)
    return 1.0 + 9.0 * np.exp(-((T - 1400.0) / 450.0) ** 2) * (T > 850.0)


def balanced_ranges(cost: Sequence[float], world: int) -> List[Tuple[int, int]]:
    """Split cells 0..n-1 into `world` contiguous [start, stop) ranges whose
    cost sums are as equal as the prefix split allows.  Every range is
    non-overlapping and together they cover all cells; ranges may be empty
    when there are fewer cells than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    c = np.asarray(cost, dtype=np.float64)
    n = c.size
    if n == 0:
        return [(0, 0)] * world
    if np.any(c < 0) or not np.all(np.isfinite(c)):
        raise ValueError("costs must be finite and non-negative")
    prefix = np.concatenate([[0.0], np.cumsum(c)])
    total = prefix[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(prefix, target, side="left"))
        b = min(max(b, bounds[-1]), n)
        bounds.append(b)
    bounds.append(n)
    return [(bounds[r], bounds[r + 1]) for r in range(world)]


def rank_range(T: np.ndarray, world: int, rank: int, cost: Optional[np.ndarray] = None) -> Tuple[int, int]:
    """This rank's [start, stop) of a batch every rank holds identically, from
    the batch's own data alone (no communication): cost-balanced contiguous
    ranges by the temperature proxy, or by `cost` when given."""
    ranges = balanced_ranges(temperature_cost(T) if cost is None else cost, world)
    return ranges[rank]


def shard_of(ranges: List[Tuple[int, int]], rank: int) -> slice:
    a, b = ranges[rank]
    return slice(a, b)


def integrate_shard(rank: int, world: int, T: np.ndarray, Y: np.ndarray, P, dt: float,
                    integrate: Callable[[np.ndarray, np.ndarray, object, float], np.ndarray],
                    cost: Optional[np.ndarray] = None):
    """Integrate this rank's range of a batch held (identically) by every rank.

    T[n] and Y[nsp, n] (SoA) are the whole batch; `integrate(T_part, Y_part,
    P_part, dt)` advances a contiguous part in place and returns its per-cell
    status.  Returns (slice, T_part, Y_part, status_part)."""
    n = T.size
    sl = slice(*rank_range(T, world, rank, cost))
    Tp = np.ascontiguousarray(T[sl].copy())
    Yp = np.ascontiguousarray(Y[:, sl].copy())
    Pp = P if np.ndim(P) == 0 else np.ascontiguousarray(np.asarray(P)[sl])
    st = integrate(Tp, Yp, Pp, dt) if Tp.size else np.zeros(0, dtype=np.int32)
    assert sl.stop - sl.start == Tp.size <= n
    return sl, Tp, Yp, np.asarray(st, dtype=np.int32)


def gather_to(root: int, sl: slice, Tp: np.ndarray, Yp: np.ndarray, st: np.ndarray, n: int, group=None):
    """Collect every rank's part on `root` (torch.distributed gather of Python
    objects; any backend).  Returns (T, Y, status) for the whole batch on root,
    None elsewhere."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world if dist.get_rank(group) == root else None
    dist.gather_object((sl.start, sl.stop, Tp, Yp, st), parts, dst=root, group=group)
    if parts is None:
        return None
    nsp = Yp.shape[0]
    T = np.empty(n)
    Y = np.empty((nsp, n))
    status = np.empty(n, dtype=np.int32)
    covered = np.zeros(n, dtype=bool)
    for a, b, t, y, s in parts:
        assert not covered[a:b].any(), "overlapping shards"
        covered[a:b] = True
        T[a:b], Y[:, a:b], status[a:b] = t, y, s
    assert covered.all(), "shards do not cover the batch"
    return T, Y, status

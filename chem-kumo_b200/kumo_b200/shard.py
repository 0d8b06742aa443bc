"""One grid over several GPUs: contiguous ranges of 128-point blocks per rank,
evaluated independently (the blocks of chem-kumo's for_each_point_block,
src/parallel_blocks.hpp:100-168, need no exchange) and gathered on the host.
There is no collective on the data path: the only communication is the
final gather of each rank's disjoint output slice and the max-over-ranks of
a time.

Every rank evaluates its range as explicit points computed in the device's
arithmetic (origin + ((s_a i + s_b j) + s_c k), the order of the device's
grid points), so the point path gives the same values as a one-GPU
evaluation of the whole grid.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np

BLOCK = 128


def block_range(npoints: int, rank: int, world: int, block: int = BLOCK) -> Tuple[int, int]:
    """(first point, point count) of this rank: whole blocks, the first
    ``nblocks % world`` ranks one block more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank or world size")
    nblocks = (npoints + block - 1) // block
    base, extra = divmod(nblocks, world)
    first_block = rank * base + min(rank, extra)
    count_blocks = base + (1 if rank < extra else 0)
    first = min(first_block * block, npoints)
    end = min((first_block + count_blocks) * block, npoints)
    return first, end - first


def slab_range(counts: Sequence[int], rank: int, world: int, block: int = BLOCK) -> Tuple[int, int]:
    """Planes [i0, i1) of the grid's first (slowest) axis for this rank: the
    planes split as evenly as whole planes allow, the first ``nx % world``
    ranks one plane more.  A slab is a grid of its own, so each rank can
    evaluate it as a grid (and the mixed form as compact tiles).  When a
    plane holds a whole number of ``block``-point blocks (ny * nz % block ==
    0) the slab boundaries fall on block boundaries of the whole grid."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("invalid rank or world size")
    nx = int(counts[0])
    base, extra = divmod(nx, world)
    i0 = rank * base + min(rank, extra)
    return i0, i0 + base + (1 if rank < extra else 0)


def slab_grid(origin: Sequence[float], steps: np.ndarray, counts: Sequence[int], i0: int, i1: int):
    """(origin, steps, counts) of planes i0 .. i1-1 as a grid of their own;
    its points are those of the whole grid up to the rounding of the shifted
    origin (origin + i0 * step of the first axis)."""
    s = np.asarray(steps, dtype=float)
    o = np.asarray(origin, dtype=float) + s[:, 0] * i0
    return o, s, (i1 - i0, int(counts[1]), int(counts[2]))


def grid_points(origin: Sequence[float], steps: np.ndarray, counts: Sequence[int], first: int, count: int) -> np.ndarray:
    """Points first .. first+count-1 of a grid (Field order, k fastest), (count, 3)."""
    ny, nz = int(counts[1]), int(counts[2])
    q = np.arange(first, first + count, dtype=np.int64)
    i, j, k = (q // (ny * nz)).astype(float), ((q // nz) % ny).astype(float), (q % nz).astype(float)
    s = np.asarray(steps, dtype=float)
    pts = np.empty((count, 3))
    for a in range(3):
        pts[:, a] = origin[a] + ((s[a, 0] * i + s[a, 1] * j) + s[a, 2] * k)
    return pts


def gather_slices(local: List[np.ndarray], npoints: int, first: int, dist, rank: int, world: int,
                  dst: int = 0) -> List[np.ndarray]:
    """Host gather of each rank's slice (channels x count per property) into
    full arrays on rank ``dst`` (an empty list elsewhere).  Every rank calls
    ``gather_object`` with (first, arrays); only ``dst`` receives the slices."""
    parts = [None] * world if rank == dst else None
    dist.gather_object((first, [np.ascontiguousarray(a) for a in local]), parts, dst=dst)
    if rank != dst:
        return []
    out = [np.empty((a.shape[0], npoints)) for a in local]
    for f, arrays in parts:
        for o, a in zip(out, arrays):
            o[:, f:f + a.shape[1]] = a
    return out


def evaluate_grid_sharded(evaluate_points: Callable[[np.ndarray], List[np.ndarray]], origin, steps, counts,
                          dist, rank: int, world: int) -> List[np.ndarray]:
    """Evaluate this rank's block range with ``evaluate_points(points (n, 3))``
    (per property, channels x n) and gather the grid on rank 0."""
    npoints = int(np.prod(counts))
    first, count = block_range(npoints, rank, world)
    local = evaluate_points(grid_points(origin, steps, counts, first, count))
    return gather_slices(local, npoints, first, dist, rank, world)


def max_over_ranks(x: float, dist, world: int, device: str = "cpu") -> float:
    """The largest value of ``x`` over the ranks (timings are reported as the
    slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())

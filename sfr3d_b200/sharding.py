"""Independent systems across GPUs: one process per GPU, each solving its
share of the systems in one batched launch.

Many uneven systems (the batched workload) are independent, so a multi-GPU
run partitions them with no collective on the data path: each rank builds
one `GpuBatch` of its share, and the results meet on rank 0 only at the end
(`gather`).  The reference runs one system per process group under MPI
(Cg.c:256-442, ParallelMpi.c:3346) and has no batch of independent systems.

`plan` is deterministic (every rank computes the same assignment from the
same inputs without communicating): longest-processing-time first, each
system to the least-loaded rank, ties to the lower rank.
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def estimated_work(rows: int, nnz: int, iterations: float | None = None) -> float:
    """Work of one solve: bytes per iteration (FP64 SpMV + vector updates,
    12 nnz + 112 rows) times the iteration estimate (the cube root of the
    rows, the growth of Jacobi-PCG on a 3-D Poisson box, when not given)."""
    it = iterations if iterations is not None else max(1.0, rows ** (1.0 / 3.0))
    return (12.0 * nnz + 112.0 * rows) * it


def plan(work: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the systems each of `world` ranks solves, in increasing
    index order within a rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    for w in work:
        if not (w >= 0.0):
            raise ValueError("work must be non-negative and finite")
    heap = [(0.0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(work)), key=lambda i: (-work[i], i))
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + work[i], r))
    return [sorted(s) for s in shares]


def loads(work: Sequence[float], shares: Sequence[Sequence[int]]) -> list[float]:
    return [sum(work[i] for i in s) for s in shares]


def solve_share(systems, share: Sequence[int],
                solve: Callable[[list], list]) -> list[tuple[int, object]]:
    """Run `solve` on this rank's systems; returns (index, result) pairs."""
    mine = [systems[i] for i in share]
    out = solve(mine) if mine else []
    if len(out) != len(mine):
        raise RuntimeError("solve returned a result count different from its systems")
    return list(zip(share, out))


def gather(pairs: list[tuple[int, object]], count: int, group=None):
    """Collect every rank's (index, result) pairs on rank 0, ordered by
    system index (None on the other ranks).  Uses torch.distributed's
    object gather, so it works on NCCL and gloo groups alike."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    box = [None] * world if rank == 0 else None
    dist.gather_object(pairs, box, dst=0, group=group)
    if rank != 0:
        return None
    res = [None] * count
    seen = 0
    for part in box:
        for i, r in part:
            if res[i] is not None:
                raise RuntimeError(f"system {i} solved twice")
            res[i] = r
            seen += 1
    if seen != count:
        raise RuntimeError(f"{count - seen} systems missing from the gather")
    return res

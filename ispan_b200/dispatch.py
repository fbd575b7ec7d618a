"""Sharding independent graphs over GPUs (one process per GPU).

Graphs are independent units, so the multi-GPU form of the batched and
served paths has no data-path collective: a host dispatcher assigns whole
graphs to ranks within each rank's device-memory budget, every rank solves
its own share in one batched call, and the labels are gathered on one rank.
The reference has no multi-graph or multi-GPU form of this path (its
src_mpi/ variant partitions one graph; that scheme is not used here).

``assign_graphs`` is a pure function (deterministic, so every rank computes
the same assignment without a message); ``run_sharded`` runs on every rank of
an initialised ``torch.distributed`` group (nccl on GPUs, gloo on CPU).
"""
from __future__ import annotations

from typing import Callable, Sequence


def graph_bytes(V: int, E: int) -> int:
    """Device bytes one graph takes in a batch: its CSR in the union (int64
    offsets, int32 ids, both directions) plus the per-vertex and per-edge
    scratch of a context (about 80 B per vertex, 4 B per 2048 edges)."""
    return 2 * 8 * (V + 1) + 2 * 4 * E + 80 * V + 4 * (E // 2048 + 4)


def assign_graphs(sizes: Sequence[tuple[int, int]], world_size: int,
                  budget_bytes: int | None = None) -> list[list[int]]:
    """Assign graph indices to ranks: largest first, each to the rank with the
    least assigned bytes (ties to the lowest rank), so the slowest rank's
    share stays near the mean.  ``sizes`` holds (V, E) per graph.  Raises
    ValueError when a graph alone, or a rank's share, exceeds the budget."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    cost = [graph_bytes(V, E) for V, E in sizes]
    order = sorted(range(len(sizes)), key=lambda i: (-cost[i], i))
    load = [0] * world_size
    out: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        if budget_bytes is not None and cost[i] > budget_bytes:
            raise ValueError(f"graph {i} needs {cost[i]} bytes, above the per-rank budget {budget_bytes}")
        r = min(range(world_size), key=lambda k: (load[k], k))
        if budget_bytes is not None and load[r] + cost[i] > budget_bytes:
            raise ValueError(f"the graphs do not fit {world_size} ranks of {budget_bytes} bytes")
        load[r] += cost[i]
        out[r].append(i)
    for share in out:
        share.sort()
    return out


def run_sharded(graphs: Sequence, sizes: Sequence[tuple[int, int]], solve: Callable[[list], list],
                budget_bytes: int | None = None, dst: int = 0):
    """Solve ``graphs`` over the ranks of the default process group.

    Every rank passes the same ``graphs`` description (or a lazy handle per
    graph) and ``sizes``; rank r solves ``assign_graphs(...)[r]`` with
    ``solve(list_of_graphs) -> list_of_labels`` (for example
    ``Context.run_graphs``) and the labels are gathered on rank ``dst``, which
    returns a list indexed like ``graphs``; other ranks return None.  A rank
    that fails raises locally; the others see the gather fail with the
    group's timeout."""
    import torch.distributed as dist
    ws, rank = dist.get_world_size(), dist.get_rank()
    share = assign_graphs(sizes, ws, budget_bytes)[rank]
    labels = solve([graphs[i] for i in share]) if share else []
    mine = list(zip(share, labels))
    gathered = [None] * ws if rank == dst else None
    dist.gather_object(mine, gathered, dst=dst)
    if rank != dst:
        return None
    out = [None] * len(graphs)
    for part in gathered:
        for i, lab in part:
            out[i] = lab
    return out

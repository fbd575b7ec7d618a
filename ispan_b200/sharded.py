"""Reachability and the giant SCC over a graph whose rows are split across
GPUs (one process per GPU, torch.distributed).

For a graph larger than one GPU's memory, the reference's MPI variant
(src_mpi/) splits the vertex range across ranks and merges each BFS level's
frontier state with an all-reduce (MAX over a byte per vertex,
src_mpi/fw_bw.h:193, :309; bitwise OR over a bitmap, :382-442).  The same
scheme here: each rank holds the forward and backward CSR rows of its vertex
range (adjacency in global ids); a level is one ``ispan_shard_expand`` kernel
per rank over its owned frontier vertices, then a MAX all-reduce of the
full-length next-frontier byte map (NCCL over NVLink on GPUs, gloo on CPU),
after which every rank holds the same frontier and visited maps.

Only the search is sharded (the elephant stage); a full sharded pipeline
would also shard the trims and the small-SCC stages.  The byte maps are
plumbing held in torch tensors; the per-level work is the CUDA kernel.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check


@dataclass
class Rows:
    """CSR rows of the vertices [v0, v0 + n) of a V-vertex graph: local
    offsets (n + 1), global adjacency ids."""

    v0: int
    n: int
    beg: object
    adj: object


def split_rows(beg: np.ndarray, adj: np.ndarray, rank: int, world: int) -> Rows:
    """Rank ``rank``'s share of a CSR (host arrays): an equal vertex range."""
    V = len(beg) - 1
    v0, v1 = V * rank // world, V * (rank + 1) // world
    b = np.asarray(beg[v0:v1 + 1], np.int64)
    return Rows(v0, v1 - v0, b - b[0], np.ascontiguousarray(adj[b[0]:b[-1]], np.int32))


def to_device(rows: Rows) -> Rows:
    import torch
    return Rows(rows.v0, rows.n, torch.from_numpy(rows.beg).cuda(),
                torch.from_numpy(rows.adj if len(rows.adj) else np.zeros(1, np.int32)).cuda()[:len(rows.adj)])


def gpu_expand(rows: Rows, V: int, frontier, visited, allowed, nxt) -> None:
    """One level on this rank's rows (CUDA kernel, torch uint8 CUDA maps)."""
    g = _lib.Csr(rows.n, int(rows.adj.numel()), rows.beg.data_ptr(), rows.beg.data_ptr(), rows.adj.data_ptr(),
                 rows.adj.data_ptr(), 8, 1)
    a = None if allowed is None else C.c_void_p(allowed.data_ptr())
    check(_lib.lib().ispan_shard_expand(C.byref(g), rows.v0, V, C.c_void_p(frontier.data_ptr()),
                                        C.c_void_p(visited.data_ptr()), a, C.c_void_p(nxt.data_ptr()), None),
          "ispan_shard_expand")


def reach(rows: Rows, V: int, seeds, allowed=None, expand=gpu_expand, device=None):
    """Vertices reachable from ``seeds`` (restricted to ``allowed`` if given)
    as a uint8 map of V entries, identical on every rank."""
    import torch
    import torch.distributed as dist
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    visited = torch.zeros(V, dtype=torch.uint8, device=dev)
    frontier = torch.zeros(V, dtype=torch.uint8, device=dev)
    s = torch.as_tensor(seeds, dtype=torch.int64, device=dev)
    visited[s] = 1
    frontier[s] = 1
    distributed = dist.is_available() and dist.is_initialized()
    for _ in range(V + 1):  # every level visits a vertex; more is a bug
        nxt = torch.zeros(V, dtype=torch.uint8, device=dev)
        expand(rows, V, frontier, visited, allowed, nxt)
        if distributed:
            dist.all_reduce(nxt, op=dist.ReduceOp.MAX)
        n = int(nxt.sum())
        if n == 0:
            return visited
        visited = torch.maximum(visited, nxt)
        frontier = nxt
    raise RuntimeError("reach did not converge")


def giant_scc(fw: Rows, bw: Rows, V: int, pivot: int, expand=gpu_expand, device=None):
    """The SCC of ``pivot``: forward reach, then backward reach inside it."""
    f = reach(fw, V, [pivot], None, expand, device)
    return reach(bw, V, [pivot], f, expand, device)

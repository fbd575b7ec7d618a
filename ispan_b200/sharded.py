"""Reachability and the giant SCC over a graph whose rows are split across
GPUs (one process per GPU, torch.distributed).

For a graph larger than one GPU's memory, the reference's MPI variant
(src_mpi/) splits the vertex range across ranks and merges each BFS level's
frontier state with collectives (MAX over a byte per vertex,
src_mpi/fw_bw.h:193, :309; bitwise OR over a visited bitmap, :382-442).
Here each rank holds the forward and backward CSR rows of its vertex range
(adjacency in global ids; ranges are whole 32-vertex words) and a level is:

1. ``ispan_shard_expand_queue``: the rank's owned frontier queue marks the
   unvisited (and allowed) neighbours in a byte map of V entries;
2. a reduce-scatter (MAX) of the byte maps: each rank receives the slice of
   the merged next frontier that it owns (NCCL over NVLink, gloo on CPU);
3. ``ispan_shard_collect``: the owner keeps the vertices it has not visited,
   sets their bits and queues them for the next level;
4. an all-gather of the owned visited words (packed bits) replicates the
   visited bitmap, which step 1 reads.

The frontier count is summed on the device and read by the host only every
``check_every`` levels (levels after the search ends find empty queues and
do nothing), so the host does not wait on the GPU once per level.  Work per
level is proportional to the frontier's edges; per level and rank the
collectives move V bytes into the reduce-scatter and V/8 bytes out of the
all-gather.  Only the search is sharded (the elephant stage).
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


def words_per_rank(V: int, world: int) -> int:
    """Owned 32-vertex words per rank (the last rank's share may be short)."""
    W = (V + 31) // 32
    return max(1, (W + world - 1) // world)


def owned_range(V: int, rank: int, world: int) -> tuple[int, int]:
    S = words_per_rank(V, world)
    v0 = min(V, rank * S * 32)
    return v0, min(V, v0 + S * 32)


def split_rows(beg: np.ndarray, adj: np.ndarray, rank: int, world: int) -> Rows:
    """Rank ``rank``'s share of a CSR (host arrays): its owned vertex range."""
    V = len(beg) - 1
    v0, v1 = owned_range(V, rank, world)
    b = np.asarray(beg[v0:v1 + 1], np.int64)
    return Rows(v0, v1 - v0, b - b[0], np.ascontiguousarray(adj[b[0]:b[-1]], np.int32))


def to_device(rows: Rows) -> Rows:
    import torch
    return Rows(rows.v0, rows.n, torch.from_numpy(rows.beg).cuda(),
                torch.from_numpy(rows.adj if len(rows.adj) else np.zeros(1, np.int32)).cuda()[:len(rows.adj)])


class GpuOps:
    """The two per-level kernels of the library (torch CUDA tensors)."""

    @staticmethod
    def expand(rows: Rows, V: int, queue, qn, visited, allowed, nxt) -> None:
        g = _lib.Csr(rows.n, int(rows.adj.numel()), rows.beg.data_ptr(), rows.beg.data_ptr(), rows.adj.data_ptr(),
                     rows.adj.data_ptr(), 8, 1)
        a = None if allowed is None else C.c_void_p(allowed.data_ptr())
        check(_lib.lib().ispan_shard_expand_queue(C.byref(g), rows.v0, V, C.c_void_p(queue.data_ptr()),
                                                  C.c_void_p(qn.data_ptr()), C.c_void_p(visited.data_ptr()), a,
                                                  C.c_void_p(nxt.data_ptr()), None), "ispan_shard_expand_queue")

    @staticmethod
    def collect(v0: int, n_own: int, mine, visited, queue, qn) -> None:
        check(_lib.lib().ispan_shard_collect(v0, n_own, C.c_void_p(mine.data_ptr()), C.c_void_p(visited.data_ptr()),
                                             C.c_void_p(queue.data_ptr()), C.c_void_p(qn.data_ptr()), None),
              "ispan_shard_collect")


def gpu_expand(rows: Rows, V: int, frontier, visited, allowed, nxt) -> None:
    """The byte-map form of one level (ispan_shard_expand): every owned vertex
    set in ``frontier`` marks its unvisited, allowed neighbours in ``nxt``."""
    g = _lib.Csr(rows.n, int(rows.adj.numel()), rows.beg.data_ptr(), rows.beg.data_ptr(), rows.adj.data_ptr(),
                 rows.adj.data_ptr(), 8, 1)
    a = None if allowed is None else C.c_void_p(allowed.data_ptr())
    check(_lib.lib().ispan_shard_expand(C.byref(g), rows.v0, V, C.c_void_p(frontier.data_ptr()),
                                        C.c_void_p(visited.data_ptr()), a, C.c_void_p(nxt.data_ptr()), None),
          "ispan_shard_expand")


def bits_to_map(bits, V: int):
    """Packed visited bits (int32 words) -> uint8 map of V entries."""
    import torch
    b = bits.to(torch.int64) & 0xFFFFFFFF
    shifts = torch.arange(32, device=bits.device, dtype=torch.int64)
    return ((b[:, None] >> shifts) & 1).reshape(-1)[:V].to(torch.uint8)


def reach(rows: Rows, V: int, seeds, allowed=None, ops=GpuOps, device=None, check_every: int = 4):
    """Vertices reachable from ``seeds`` (restricted to ``allowed``, packed
    visited bits of a previous search, if given) as packed bits: int32 words
    covering V vertices, identical on every rank."""
    import torch
    import torch.distributed as dist
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if distributed else 1
    rank = dist.get_rank() if distributed else 0
    S = words_per_rank(V, world)
    v0, v1 = owned_range(V, rank, world)
    assert rows.v0 == v0 and rows.n == v1 - v0, "rows are not this rank's owned range"
    visited = torch.zeros(S * world, dtype=torch.int32, device=dev)
    nxt = torch.zeros(S * 32 * world, dtype=torch.uint8, device=dev)
    mine = torch.empty(S * 32, dtype=torch.uint8, device=dev)
    queue = torch.empty(max(1, S * 32), dtype=torch.int32, device=dev)
    qn = torch.zeros(1, dtype=torch.int64, device=dev)
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    # seeds: their bits everywhere, each in its owner's queue
    s = np.unique(np.asarray(seeds, np.int64))
    sv = np.zeros(S * world, np.uint32)
    np.bitwise_or.at(sv, s >> 5, (np.uint32(1) << (s & 31).astype(np.uint32)))
    visited.copy_(torch.from_numpy(sv.view(np.int32)))
    own = s[(s >= v0) & (s < v1)]
    queue[:len(own)] = torch.from_numpy(own.astype(np.int32)).to(dev)
    qn.fill_(len(own))
    for level in range(V + check_every + 1):  # every level visits a vertex until the search ends
        nxt.zero_()
        ops.expand(rows, V, queue, qn, visited, allowed, nxt)
        if distributed:
            dist.reduce_scatter_tensor(mine, nxt, op=dist.ReduceOp.MAX)
        else:
            mine.copy_(nxt[:S * 32])
        qn.zero_()
        ops.collect(v0, v1 - v0, mine, visited, queue, qn)
        if distributed:
            own_words = visited[rank * S:(rank + 1) * S].clone()
            dist.all_gather_into_tensor(visited, own_words)
            total.copy_(qn)
            dist.all_reduce(total, op=dist.ReduceOp.SUM)
        else:
            total.copy_(qn)
        if level % check_every == check_every - 1 and int(total.item()) == 0:
            return visited
    raise RuntimeError("reach did not converge")


def giant_scc(fw: Rows, bw: Rows, V: int, pivot: int, ops=GpuOps, device=None):
    """The SCC of ``pivot`` as a uint8 map of V entries: forward reach, then
    backward reach inside it."""
    f = reach(fw, V, [pivot], None, ops, device)
    b = reach(bw, V, [pivot], f, ops, device)
    return bits_to_map(b, V)

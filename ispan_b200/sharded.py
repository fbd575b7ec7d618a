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
all-gather.  ``scc`` runs the whole detection on such rows: trim-1 and the
pivot's SCC sharded, the residual gathered and solved on one GPU per rank.
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


# ---------------------------------------------------------------------------
# The whole detection over sharded rows: trim-1, the pivot's SCC by the
# sharded searches above, and the residual solved where it fits.
#
# The reference's MPI variant exchanges state at three points: the trim-1
# statuses after the first trim (an all-gather of each rank's range,
# src_mpi/scc_core.cpp:280-287), the labels after the giant's searches (a MAX
# all-reduce of the label array, :529-535) and the labels of the small
# components (a MAX all-reduce, :704-711).  Here the status is a packed
# bitmap of active vertices, replicated by an all-gather of each rank's owned
# words; the giant's label is a MIN all-reduce of its owned members' ids; and
# the residual -- on the graphs this form is for, a small fraction next to the
# giant -- is gathered whole to every rank and solved there by the
# single-GPU engine (every rank gets the same labels, so no label exchange
# is needed).  The per-round degree counts are tensor operations on the
# rank's own rows (any device), not a kernel of this library.

def _own_edges(rows: Rows, dev):
    """Per edge of the rank's rows: its source row (local) and target (global)."""
    import torch
    beg = torch.as_tensor(rows.beg, device=dev).to(torch.int64)  # host arrays or device tensors
    adj = torch.as_tensor(rows.adj, device=dev).to(torch.int64)
    row = torch.repeat_interleave(torch.arange(rows.n, device=dev), beg[1:] - beg[:-1])
    return row, adj


def _bit(words, ids):
    """Bits of the packed int32 words at vertex ids (int64 tensor) as bool."""
    return ((words[ids >> 5] >> (ids & 31)) & 1) != 0


def _pack(own, S: int):
    """A bool tensor of at most S * 32 owned vertices as S int32 words."""
    import torch
    b = torch.zeros(S * 32, dtype=torch.int64, device=own.device)
    b[:own.numel()] = own.to(torch.int64)
    w = (b.view(S, 32) << torch.arange(32, device=own.device)).sum(1)
    return (w - (w >= 1 << 31).to(torch.int64) * (1 << 32)).to(torch.int32)


def _allgather_words(mine, out):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.all_gather_into_tensor(out, mine.contiguous())
    else:
        out[:mine.numel()] = mine


def _allreduce(t, op):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=op)
    return t


def trim1(fw: Rows, bw: Rows, V: int, rounds: int = 3, device=None):
    """Trim-1 over sharded rows (trim_1_first, src/trim_1_gfq.h:9-33, and the
    peel rounds after it): a vertex with no active out-neighbour or no active
    in-neighbour other than itself is its own SCC.  Returns (active bits,
    trimmed bits), packed int32 words over V, identical on every rank.
    `rounds` peel rounds at most: trim-1 only takes work off the later
    stages, which find the same SCCs in what it leaves."""
    import torch
    import torch.distributed as dist
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if distributed else 1
    rank = dist.get_rank() if distributed else 0
    S = words_per_rank(V, world)
    v0, v1 = owned_range(V, rank, world)
    own = torch.ones(v1 - v0, dtype=torch.bool, device=dev)
    trimmed_own = torch.zeros(v1 - v0, dtype=torch.bool, device=dev)
    active = torch.zeros(S * world, dtype=torch.int32, device=dev)
    _allgather_words(_pack(own, S), active)
    ids = torch.arange(v0, v1, device=dev)
    ef, eb = _own_edges(fw, dev), _own_edges(bw, dev)
    for _ in range(max(0, rounds)):
        deg = []
        for row, adj in (ef, eb):
            live = _bit(active, adj) & (adj != ids[row])
            deg.append(torch.zeros(v1 - v0, dtype=torch.int64, device=dev).index_add_(0, row, live.to(torch.int64)))
        rem = own & ((deg[0] == 0) | (deg[1] == 0))
        n = _allreduce(rem.sum().reshape(1).to(torch.int64), dist.ReduceOp.SUM if distributed else None)
        if int(n.item()) == 0:
            break
        own &= ~rem
        trimmed_own |= rem
        _allgather_words(_pack(own, S), active)
    trimmed = torch.zeros(S * world, dtype=torch.int32, device=dev)
    _allgather_words(_pack(trimmed_own, S), trimmed)
    return active, trimmed


def pivot(fw: Rows, bw: Rows, V: int, active, device=None) -> int:
    """The pivot (pivot_selection_from_fq, src/scc_common.h:92-150): the active
    vertex of largest out-degree x in-degree, ties to the lowest id, as a MAX
    all-reduce of a 64-bit key; -1 when no vertex is active."""
    import torch
    import torch.distributed as dist
    dev = active.device
    v0, n = fw.v0, fw.n
    if n:
        fb = torch.as_tensor(fw.beg, device=dev).to(torch.int64)
        bb = torch.as_tensor(bw.beg, device=dev).to(torch.int64)
        od, idg = fb[1:] - fb[:-1], bb[1:] - bb[:-1]
        ids = torch.arange(v0, v0 + n, device=dev)
        key = (torch.clamp(od * idg, max=(1 << 31) - 1) << 32) | (0xFFFFFFFF - ids)
        key = torch.where(_bit(active, ids), key, torch.full_like(key, -1))
        best = key.max().reshape(1)
    else:
        best = torch.full((1,), -1, dtype=torch.int64, device=dev)
    distributed = dist.is_available() and dist.is_initialized()
    best = int(_allreduce(best, dist.ReduceOp.MAX if distributed else None).item())
    return -1 if best < 0 else 0xFFFFFFFF - (best & 0xFFFFFFFF)


def _gpu_solve(csr):
    from . import Context
    with Context(max(csr.V, 1), max(csr.E, 1)) as ctx:
        labels, _ = ctx.run_csr(csr)
    return np.asarray(labels)


def scc(fw: Rows, bw: Rows, V: int, solve=None, ops=GpuOps, device=None, trim_rounds: int = 3):
    """SCC labels (minimum member id, int64 numpy array of V) of a graph whose
    rows are sharded across the ranks, identical on every rank: sharded
    trim-1, the pivot's SCC by the sharded searches, and the residual's
    subgraph gathered to every rank and solved by `solve(csr) -> labels`
    (default: the single-GPU engine)."""
    import torch
    import torch.distributed as dist
    from . import graphs as G
    dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
    distributed = dist.is_available() and dist.is_initialized()
    world = dist.get_world_size() if distributed else 1
    solve = solve or _gpu_solve
    labels = np.arange(V, dtype=np.int64)  # trimmed vertices are their own SCC
    active, _ = trim1(fw, bw, V, trim_rounds, dev)
    p = pivot(fw, bw, V, active, dev)
    giant = torch.zeros_like(active)
    if p >= 0:
        f = reach(fw, V, [p], active, ops, dev)
        giant = reach(bw, V, [p], f, ops, dev)
        gm = bits_to_map(giant, V).to(torch.bool)
        own = gm[fw.v0:fw.v0 + fw.n]
        lo = torch.full((1,), V, dtype=torch.int64, device=dev)
        if bool(own.any()):
            lo[0] = int(torch.nonzero(own)[0, 0]) + fw.v0
        gmin = int(_allreduce(lo, dist.ReduceOp.MIN if distributed else None).item())
        labels[gm.cpu().numpy()] = gmin
    # the residual: active, outside the giant; each rank sends its rows' edges
    # between residual vertices, every rank builds and solves the subgraph
    resid = bits_to_map(active & ~giant, V).to(torch.bool)
    row, adj = _own_edges(fw, dev)
    src = row + fw.v0
    keep = resid[src] & resid[adj]
    mine = torch.stack([src[keep], adj[keep]], 1).to(torch.int64)
    if distributed:
        cnt = torch.tensor([mine.shape[0]], dtype=torch.int64, device=dev)
        cnts = [torch.zeros_like(cnt) for _ in range(world)]
        dist.all_gather(cnts, cnt)
        m = max(int(c.item()) for c in cnts)
        pad = torch.full((m, 2), -1, dtype=torch.int64, device=dev)
        pad[:mine.shape[0]] = mine
        parts = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad)
        edges = torch.cat([q[:int(c.item())] for q, c in zip(parts, cnts)])
    else:
        edges = mine
    ids = torch.nonzero(resid).flatten()
    if ids.numel():
        local = torch.searchsorted(ids, edges.reshape(-1)).reshape(-1, 2)
        sub = G.from_edges(int(ids.numel()), local.cpu().numpy())
        lab = np.asarray(solve(sub), np.int64)
        labels[ids.cpu().numpy()] = ids.cpu().numpy()[lab]  # order-preserving ids: minima map to minima
    return labels

"""The per-level kernels of the sharded search on the GPU
(ispan_shard_expand_queue, ispan_shard_collect): one rank alone, and four
shards on one device with the reduce-scatter and all-gather carried out by
tensor operations, both give the pivot's exact SCC; the byte-map form
(ispan_shard_expand) as well."""
import numpy as np
import pytest
import torch

import oracle
from ispan_b200 import graphs as G
from ispan_b200.sharded import (GpuOps, bits_to_map, giant_scc, gpu_expand, owned_range, split_rows, to_device,
                                words_per_rank)

pytestmark = pytest.mark.gpu


def _case():
    g = G.rmat(13, 8, 6)
    exact = oracle.tarjan(g)
    vals, counts = np.unique(exact, return_counts=True)
    return g, exact, int(vals[np.argmax(counts)])


def test_single_rank_gpu_search():
    g, exact, p = _case()
    fw = to_device(split_rows(g.fw_beg, g.fw_adj, 0, 1))
    bw = to_device(split_rows(g.bw_beg, g.bw_adj, 0, 1))
    s = giant_scc(fw, bw, g.V, p).cpu().numpy().astype(bool)
    assert np.array_equal(s, exact == exact[p])


def _reach_shards(shards, V, seeds, allowed, world):
    """The distributed level loop of ispan_b200.sharded.reach with `world`
    ranks on one GPU: each rank's kernels on its own queue, the
    reduce-scatter as a MAX over the ranks' maps sliced by owner, the
    all-gather as the owners' words copied into one bitmap."""
    S = words_per_rank(V, world)
    s = np.asarray(seeds, np.int64)
    words = np.zeros(S * world, np.uint32)
    np.bitwise_or.at(words, s >> 5, np.uint32(1) << (s & 31).astype(np.uint32))
    vis = torch.from_numpy(words.view(np.int32)).cuda()
    queues, qns = [], []
    for r in range(world):
        v0, v1 = owned_range(V, r, world)
        own = s[(s >= v0) & (s < v1)]
        q = torch.zeros(S * 32, dtype=torch.int32, device="cuda")
        q[:len(own)] = torch.from_numpy(own.astype(np.int32)).cuda()
        queues.append(q)
        qns.append(torch.tensor([len(own)], dtype=torch.int64, device="cuda"))
    for _ in range(V + 1):
        maps = []
        for r in range(world):
            m = torch.zeros(S * 32 * world, dtype=torch.uint8, device="cuda")
            GpuOps.expand(shards[r], V, queues[r], qns[r], vis, allowed, m)
            maps.append(m)
        merged = torch.stack(maps).amax(0)
        new = vis.clone()
        for r in range(world):
            v0, v1 = owned_range(V, r, world)
            mine = merged[r * S * 32:(r + 1) * S * 32].contiguous()
            qns[r].zero_()
            own = vis.clone()  # each rank updates its own copy; the owners' words are gathered below
            GpuOps.collect(v0, v1 - v0, mine, own, queues[r], qns[r])
            new[r * S:(r + 1) * S] = own[r * S:(r + 1) * S]
        vis = new
        if sum(int(q.item()) for q in qns) == 0:
            return vis
    raise RuntimeError("no convergence")


def test_four_shards_merged_like_the_collectives():
    g, exact, p = _case()
    shards_fw = [to_device(split_rows(g.fw_beg, g.fw_adj, r, 4)) for r in range(4)]
    shards_bw = [to_device(split_rows(g.bw_beg, g.bw_adj, r, 4)) for r in range(4)]
    f = _reach_shards(shards_fw, g.V, [p], None, 4)
    b = _reach_shards(shards_bw, g.V, [p], f, 4)
    assert np.array_equal(bits_to_map(b, g.V).cpu().numpy().astype(bool), exact == exact[p])


def test_byte_map_form():
    """ispan_shard_expand (the byte-map form) level by level on one rank."""
    g, exact, p = _case()
    fw = to_device(split_rows(g.fw_beg, g.fw_adj, 0, 1))
    V = g.V
    visited = torch.zeros(V, dtype=torch.uint8, device="cuda")
    frontier = torch.zeros(V, dtype=torch.uint8, device="cuda")
    visited[p] = 1
    frontier[p] = 1
    for _ in range(V + 1):
        nxt = torch.zeros(V, dtype=torch.uint8, device="cuda")
        gpu_expand(fw, V, frontier, visited, None, nxt)
        if int(nxt.sum()) == 0:
            break
        visited = torch.maximum(visited, nxt)
        frontier = nxt
    # forward set of the pivot by a CPU BFS
    want = np.zeros(V, bool)
    want[p] = True
    stack = [p]
    while stack:
        v = stack.pop()
        for w in g.fw_adj[g.fw_beg[v]:g.fw_beg[v + 1]]:
            if not want[w]:
                want[w] = True
                stack.append(w)
    assert np.array_equal(visited.cpu().numpy().astype(bool), want)

"""The per-rank kernel of the sharded search (ispan_shard_expand) on the GPU:
rows split into several shards and merged on one rank as the all-reduce
would, and the single-rank search, both give the pivot's exact SCC."""
import numpy as np
import pytest
import torch

import oracle
from ispan_b200 import graphs as G
from ispan_b200.sharded import giant_scc, gpu_expand, split_rows, to_device

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


def test_four_shards_merged_like_the_all_reduce():
    g, exact, p = _case()
    shards_fw = [to_device(split_rows(g.fw_beg, g.fw_adj, r, 4)) for r in range(4)]
    shards_bw = [to_device(split_rows(g.bw_beg, g.bw_adj, r, 4)) for r in range(4)]

    def expand_all(shards):
        def f(rows, V, frontier, visited, allowed, nxt):
            parts = []
            for sh in shards:  # each rank's kernel into its own map, then MAX
                m = torch.zeros_like(nxt)
                gpu_expand(sh, V, frontier, visited, allowed, m)
                parts.append(m)
            nxt.copy_(torch.stack(parts).amax(0))
        return f

    from ispan_b200.sharded import reach
    f = reach(shards_fw[0], g.V, [p], None, expand_all(shards_fw))
    b = reach(shards_bw[0], g.V, [p], f, expand_all(shards_bw))
    assert np.array_equal(b.cpu().numpy().astype(bool), exact == exact[p])

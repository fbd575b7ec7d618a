"""Condensation (the SCC DAG) from the GPU labels, against the oracle's:
the distinct crossing label pairs, sorted, and acyclic."""
import numpy as np
import pytest

import oracle
from ispan_b200 import Context, condensation, graphs as G

pytestmark = pytest.mark.gpu


def expected_pairs(csr, labels):
    src = np.repeat(np.arange(csr.V), np.diff(csr.fw_beg.astype(np.int64)))
    lu, lv = labels[src], labels[csr.fw_adj]
    keep = lu != lv
    pairs = np.unique(np.stack([lu[keep], lv[keep]], 1).astype(np.int64), axis=0)
    return pairs


def is_acyclic(pairs, nodes):
    idx = {v: i for i, v in enumerate(nodes)}
    indeg = np.zeros(len(nodes), np.int64)
    out = [[] for _ in nodes]
    for a, b in pairs:
        out[idx[a]].append(idx[b])
        indeg[idx[b]] += 1
    stack = [i for i in range(len(nodes)) if indeg[i] == 0]
    seen = 0
    while stack:
        i = stack.pop()
        seen += 1
        for j in out[i]:
            indeg[j] -= 1
            if indeg[j] == 0:
                stack.append(j)
    return seen == len(nodes)


@pytest.mark.parametrize("make", [lambda: G.toy(), lambda: G.rmat(12, 8, 4), lambda: G.planted(5000, 3, giant_frac=0.2),
                                  lambda: G.random_graph(400, 2000, 5), lambda: G.from_edges(5, np.zeros((0, 2), np.int64)),
                                  lambda: G.rmat(11, 16, 6, offset_dtype=np.int64)])
def test_condensation_matches_oracle(make):
    import torch
    csr = make()
    exact = oracle.tarjan(csr)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    fb, fa = t(csr.fw_beg), t(csr.fw_adj if csr.E else np.zeros(1, np.int32))[:csr.E]
    bb, ba = t(csr.bw_beg), t(csr.bw_adj if csr.E else np.zeros(1, np.int32))[:csr.E]
    with Context(max(csr.V, 1), max(csr.E, 1)) as ctx:
        lab, _ = ctx.run(fb, fa, bb, ba)
    assert np.array_equal(lab.cpu().numpy(), exact)
    got = condensation(fb, fa, lab)
    want = expected_pairs(csr, exact)
    assert np.array_equal(got, want.reshape(-1, 2))
    assert is_acyclic(got, np.unique(exact))

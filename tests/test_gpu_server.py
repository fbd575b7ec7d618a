"""Batched-over-separate-graphs and served forms: every graph's labels in a
batch or in the server's mix are those of the graph run alone, which are the
oracle's exact SCC partition (min-id labels)."""
import numpy as np
import pytest

import oracle
from ispan_b200 import Context, IspanError, Server, graphs as G

pytestmark = pytest.mark.gpu


def _mix(seed=0):
    """A seeded mix of shapes and offset widths, including edge cases."""
    gs = [G.toy(), G.rmat(10, 16, seed + 1), G.planted(3000, seed + 2, giant_frac=0.3),
          G.planted(20000, seed + 3, giant_frac=0.0, dag_ef=3.0, max_cycle=300),
          G.random_graph(500, 3000, seed + 4), G.rmat(12, 8, seed + 5, offset_dtype=np.int64),
          G.from_edges(7, np.zeros((0, 2), np.int64)),           # no edges
          G.from_edges(1, np.zeros((0, 2), np.int64)),           # one vertex
          G.planted(800, seed + 6, giant_frac=0.9)]
    return gs


def _dev(csr):
    import torch
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t(csr.fw_beg), t(csr.fw_adj if csr.E else np.zeros(1, np.int32))[:csr.E], t(csr.bw_beg), \
        t(csr.bw_adj if csr.E else np.zeros(1, np.int32))[:csr.E]


@pytest.fixture(scope="module")
def ctx():
    c = Context(1 << 20, 1 << 23)
    yield c
    c.close()


def test_run_graphs_host_and_device_mixed(ctx):
    gs = _mix(0)
    arrays = []
    for i, g in enumerate(gs):  # alternate host and device graphs
        arrays.append((g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj) if i % 2 == 0 else _dev(g))
    labels, st = ctx.run_graphs(arrays)
    total = 0
    for g, lab in zip(gs, labels):
        lab = lab.cpu().numpy() if hasattr(lab, "cpu") else lab
        exact = oracle.tarjan(g)
        assert np.array_equal(lab, exact)
        total += oracle.scc_count(exact)
    assert st["scc_count"] == total


def test_run_graphs_same_as_alone_twice(ctx):
    gs = _mix(7)
    alone = [ctx.run_csr(g)[0].copy() for g in gs]
    for _ in range(2):
        labels, _ = ctx.run_graphs([(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj) for g in gs])
        for a, b in zip(alone, labels):
            assert np.array_equal(a, b)


def test_run_graphs_rejects_bad_graph(ctx):
    import torch
    g = G.rmat(8, 4, 3)
    bad_adj = g.fw_adj.copy()
    bad_adj[5] = g.V + 3  # id out of range: the pack kernel refuses the batch
    fb, fa, bb, ba = _dev(g)
    with pytest.raises(IspanError) as e:
        ctx.run_graphs([(fb, torch.from_numpy(bad_adj).cuda(), bb, ba), _dev(G.toy())])
    assert e.value.code == -1
    off = g.fw_beg.copy()
    assert off[4] + 1 <= g.E
    off[3] = off[4] + 1  # offsets decrease from vertex 3 to 4
    with pytest.raises(IspanError):
        ctx.run_graphs([(torch.from_numpy(off).cuda(), fa, bb, ba)])
    # the context still works afterwards
    labels, _ = ctx.run_graphs([_dev(G.toy())])
    assert np.array_equal(labels[0].cpu().numpy(), oracle.tarjan(G.toy()))


def test_server_mix_equals_alone():
    """Requests served in batches with other graphs give the labels of the
    graph run alone."""
    import torch
    pool = _mix(3) + _mix(11)
    with Context(1 << 20, 1 << 23) as c:
        alone = [c.run_csr(g)[0].copy() for g in pool]
    rng = np.random.default_rng(5)
    order = rng.integers(0, len(pool), size=120)
    with Server(max_batch_graphs=16, hbm_budget_bytes=8 << 30) as srv:
        maxV, maxE, maxN = srv.limits()
        assert maxN == 16 and maxV > 0 and maxE > 0
        dev = [_dev(g) for g in pool]
        outs, tickets = [], []
        for k, i in enumerate(order):
            if k % 3 == 0:  # host request, host labels
                g = pool[i]
                out = np.full(max(g.V, 1), -7, np.int32)
                tickets.append(srv.submit(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, out))
            else:           # device request, device labels
                out = torch.full((max(pool[i].V, 1),), -7, dtype=torch.int32, device="cuda")
                tickets.append(srv.submit(*dev[i], out))
            outs.append(out)
        infos = [srv.wait(t, timeout_s=120) for t in tickets]
        assert all(inf is not None and inf["status"] == 1 for inf in infos)
        assert max(inf["batch_graphs"] for inf in infos) > 1  # really served in a mix
        for i, out, inf in zip(order, outs, infos):
            got = out.cpu().numpy() if hasattr(out, "cpu") else out
            assert np.array_equal(got[:pool[i].V], alone[i]), f"request of graph {i} in batch {inf['batch_id']}"
        cnt = srv.counters()
        assert cnt["graphs"] == len(order) and cnt["queued"] == 0
        with pytest.raises(IspanError):  # a finished request is reported once
            srv.poll(tickets[0])


def test_server_refuses_oversize_request():
    with Server(max_batch_graphs=4, max_batch_V=1000, max_batch_E=10000, hbm_budget_bytes=1 << 30) as srv:
        g = G.rmat(12, 8, 1)
        out = np.empty(g.V, np.int32)
        with pytest.raises(IspanError) as e:
            srv.submit(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, out)
        assert e.value.code == -7
        t = G.toy()
        o = np.empty(t.V, np.int32)
        tk = srv.submit(t.fw_beg, t.fw_adj, t.bw_beg, t.bw_adj, o)
        assert srv.wait(tk, 60)["status"] == 1
        assert np.array_equal(o, oracle.tarjan(t))

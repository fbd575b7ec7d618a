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
    # host graphs are checked on the device the same way: falling offsets,
    # offsets that do not end at E, ids out of range
    end = g.bw_beg.copy()
    end[-1] -= 1
    for host in ((off, g.fw_adj, g.bw_beg, g.bw_adj), (g.fw_beg, g.fw_adj, end, g.bw_adj),
                 (g.fw_beg, bad_adj, g.bw_beg, g.bw_adj)):
        with pytest.raises(IspanError) as e:
            ctx.run_graphs([host, (G.toy().fw_beg, G.toy().fw_adj, G.toy().bw_beg, G.toy().bw_adj)])
        assert e.value.code == -1
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
    """A request whose footprint exceeds the whole budget is refused at
    submission; smaller ones are served."""
    with Server(max_batch_graphs=4, max_batch_V=1000, max_batch_E=10000, hbm_budget_bytes=16 << 20) as srv:
        g = G.from_edges(300_000, np.zeros((0, 2), np.int64))  # ~100 B of scratch per vertex > 16 MiB
        out = np.empty(g.V, np.int32)
        with pytest.raises(IspanError) as e:
            srv.submit(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, out)
        assert e.value.code == -7
        t = G.toy()
        o = np.empty(t.V, np.int32)
        tk = srv.submit(t.fw_beg, t.fw_adj, t.bw_beg, t.bw_adj, o)
        assert srv.wait(tk, 60)["status"] == 1
        assert np.array_equal(o, oracle.tarjan(t))


def _slow_graph():
    """A 1e6-vertex random DAG of planted cycles (lengths up to 1000): its
    colouring rounds keep a lane busy for a long time."""
    import torch
    from ispan_b200 import gen
    g = gen.batch(nseg=2, vmin=1_000_000, vmax=1_000_000, ef_min=8, ef_max=8, max_cycle=1000, seed=5)
    fb, fa, bb, ba = g.extract(1, "int64")  # odd graphs of a batch are the planted DAGs
    g.free()
    torch.cuda.synchronize()
    host = G.CSR(int(fb.numel()) - 1, int(fa.numel()), fb.cpu().numpy(), fa.cpu().numpy(), bb.cpu().numpy(),
                 ba.cpu().numpy())
    return (fb, fa, bb, ba), host


def test_server_overlaps_requests_that_arrive_mid_batch():
    """Continuous batching: requests submitted while a long batch is on the
    GPU are admitted by free lanes and finish before that batch does, and
    every request's labels are those of its graph run alone (the exact
    partition)."""
    import time
    import torch
    dev, host = _slow_graph()
    small = [G.rmat(10, 16, 3), G.planted(3000, 4, giant_frac=0.3), G.toy(), G.random_graph(500, 2000, 1)]
    with Server(n_slots=4, hbm_budget_bytes=8 << 30) as srv:
        out_big = torch.full((host.V,), -7, dtype=torch.int32, device="cuda")
        tb = srv.submit(*dev, out_big)
        t_wait = time.monotonic() + 60
        while True:  # until the big request's batch is admitted (it is then on the GPU)
            info = srv.peek(tb)
            if info["t_start_ns"] > 0 or time.monotonic() > t_wait:
                break
            time.sleep(0.001)
        assert info["status"] == 0, "the long batch finished before the small requests could be sent"
        outs, tks = [], []
        for g in small:
            o = np.full(max(g.V, 1), -7, np.int32)
            tks.append(srv.submit(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, o))
            outs.append(o)
        small_info = [srv.wait(t, timeout_s=120) for t in tks]
        still_running = srv.peek(tb)["status"] == 0
        big = srv.wait(tb, timeout_s=300)
        assert big["status"] == 1 and all(i["status"] == 1 for i in small_info)
        assert still_running, "the small requests did not finish while the long batch ran"
        for i in small_info:
            assert i["batch_id"] != big["batch_id"] and i["t_done_ns"] < big["t_done_ns"]
            assert i["t_start_ns"] < big["t_done_ns"]  # admitted while the long batch ran
        for g, o in zip(small, outs):
            assert np.array_equal(o[:g.V], oracle.tarjan(g))
        assert np.array_equal(out_big.cpu().numpy(), oracle.tarjan(host))
        cnt = srv.counters()
        assert cnt["bytes_in_use"] == 0 and 0 < cnt["bytes_peak"] <= 8 << 30
        assert cnt["lane_ns"] > cnt["busy_ns"]  # more than one batch was in flight at times


def test_server_single_lane_and_memory_wait():
    """One lane, and a budget that holds one batch at a time: requests wait
    for memory, then run; labels are exact."""
    pool = _mix(5)
    with Server(n_slots=1, max_batch_graphs=2, hbm_budget_bytes=64 << 20) as srv:
        outs = [np.full(max(g.V, 1), -7, np.int32) for g in pool]
        tks = [srv.submit(g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj, o) for g, o in zip(pool, outs)]
        infos = [srv.wait(t, timeout_s=120) for t in tks]
        assert all(i["status"] == 1 for i in infos)
        for g, o in zip(pool, outs):
            assert np.array_equal(o[:g.V], oracle.tarjan(g))
        cnt = srv.counters()
        assert cnt["lanes"] == 1 and cnt["bytes_peak"] <= 64 << 20 and cnt["bytes_in_use"] == 0

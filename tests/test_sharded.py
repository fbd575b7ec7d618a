"""Sharded search (rows of one graph split across ranks), world size 2 over
gloo on CPU: the per-level merge by MAX all-reduce gives every rank the
pivot's exact SCC.  The oracle's CPU expansion stands in for the per-rank
GPU kernel (tested on the GPU in test_gpu_sharded.py)."""
import datetime
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from ispan_b200 import graphs as G
from ispan_b200.sharded import giant_scc, reach, split_rows


def cpu_expand(rows, V, frontier, visited, allowed, nxt):
    f = frontier.numpy()
    vis = visited.numpy()
    al = None if allowed is None else allowed.numpy()
    out = nxt.numpy()
    for i in np.nonzero(f[rows.v0:rows.v0 + rows.n])[0]:
        for w in rows.adj[rows.beg[i]:rows.beg[i + 1]]:
            if not vis[w] and (al is None or al[w]):
                out[w] = 1


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _graph():
    return G.planted(4000, 5, giant_frac=0.4)


def _pivot(g, exact):
    vals, counts = np.unique(exact, return_counts=True)
    return int(vals[np.argmax(counts)])  # the smallest vertex of the largest SCC


def _graph_rmat():
    return G.rmat(11, 8, 5)


def _worker(rank, world, port, q, kind="planted"):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        g = _graph() if kind == "planted" else _graph_rmat()
        exact = oracle.tarjan(g)
        p = _pivot(g, exact)
        fw = split_rows(g.fw_beg, g.fw_adj, rank, world)
        bw = split_rows(g.bw_beg, g.bw_adj, rank, world)
        s = giant_scc(fw, bw, g.V, p, expand=cpu_expand, device="cpu").numpy().astype(bool)
        q.put((rank, bool(np.array_equal(s, exact == exact[p]))))
    except Exception as e:  # noqa: BLE001
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _run_world(world, kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q, kind)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        if p.is_alive():
            p.kill()
    return sorted(q.get() for _ in range(q.qsize()))


def test_sharded_giant_world_size_2():
    res = _run_world(2, "planted")
    assert res == [(0, True), (1, True)], res


def test_sharded_giant_world_size_3_uneven_rows():
    # 2048 vertices over 3 ranks: ranges of 682, 683 and 683 rows
    res = _run_world(3, "rmat")
    assert res == [(0, True), (1, True), (2, True)], res


def test_split_rows_reassembles_the_csr():
    g = _graph_rmat()
    for world in (1, 2, 3, 5):
        parts = [split_rows(g.fw_beg, g.fw_adj, r, world) for r in range(world)]
        assert [p.v0 for p in parts] == [g.V * r // world for r in range(world)]
        assert sum(p.n for p in parts) == g.V
        adj = np.concatenate([p.adj for p in parts])
        assert np.array_equal(adj, g.fw_adj)
        deg = np.concatenate([np.diff(p.beg) for p in parts])
        assert np.array_equal(deg, np.diff(g.fw_beg))
    # more ranks than vertices: empty ranges are valid shards
    tiny_beg, tiny_adj = np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32)
    parts = [split_rows(tiny_beg, tiny_adj, r, 4) for r in range(4)]
    assert [p.n for p in parts] == [0, 1, 0, 1]
    assert np.array_equal(np.concatenate([p.adj for p in parts]), tiny_adj)


def test_allowed_map_restricts_the_search():
    g = _graph()
    exact = oracle.tarjan(g)
    p = _pivot(g, exact)
    fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
    full = reach(fw, g.V, [p], None, expand=cpu_expand, device="cpu")
    allowed = torch.from_numpy((exact == exact[p]).astype(np.uint8))
    inside = reach(fw, g.V, [p], allowed, expand=cpu_expand, device="cpu")
    assert int(inside.sum()) == int((exact == exact[p]).sum())  # an SCC is closed under reach inside it
    assert int(full.sum()) >= int(inside.sum())


def test_single_rank_matches_oracle():
    g = _graph()
    exact = oracle.tarjan(g)
    p = _pivot(g, exact)
    fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
    bw = split_rows(g.bw_beg, g.bw_adj, 0, 1)
    s = giant_scc(fw, bw, g.V, p, expand=cpu_expand, device="cpu").numpy().astype(bool)
    assert np.array_equal(s, exact == exact[p])

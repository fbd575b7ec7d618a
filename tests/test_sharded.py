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
from ispan_b200.sharded import giant_scc, split_rows


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


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        g = _graph()
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


def test_sharded_giant_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        if p.is_alive():
            p.kill()
    res = sorted(q.get() for _ in range(q.qsize()))
    assert res == [(0, True), (1, True)], res


def test_single_rank_matches_oracle():
    g = _graph()
    exact = oracle.tarjan(g)
    p = _pivot(g, exact)
    fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
    bw = split_rows(g.bw_beg, g.bw_adj, 0, 1)
    s = giant_scc(fw, bw, g.V, p, expand=cpu_expand, device="cpu").numpy().astype(bool)
    assert np.array_equal(s, exact == exact[p])

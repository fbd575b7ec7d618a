"""Sharded search and detection (rows of one graph split across ranks), world
sizes 2 and 3 over gloo on CPU: the per-level merge gives every rank the
pivot's exact SCC, and the whole detection (sharded trim-1 and pivot, the
giant, the residual gathered and solved) gives every rank the exact labels.
The oracle's CPU expansion stands in for the per-rank GPU kernels (tested on
the GPU in test_gpu_sharded.py) and the oracle's Tarjan for the single-GPU
solve of the residual."""
import datetime
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from ispan_b200 import graphs as G
from ispan_b200.sharded import bits_to_map, giant_scc, owned_range, pivot, reach, scc, split_rows, trim1


class CpuOps:
    """CPU stand-ins for the two per-level kernels (ispan_shard_expand_queue,
    ispan_shard_collect), same contract, on CPU tensors."""

    @staticmethod
    def expand(rows, V, queue, qn, visited, allowed, nxt):
        vis = visited.numpy().view(np.uint32)
        al = None if allowed is None else allowed.numpy().view(np.uint32)
        out = nxt.numpy()
        for v in queue.numpy()[:int(qn.item())]:
            i = int(v) - rows.v0
            for w in rows.adj[rows.beg[i]:rows.beg[i + 1]]:
                b = np.uint32(1) << np.uint32(w & 31)
                if not (vis[w >> 5] & b) and (al is None or (al[w >> 5] & b)):
                    out[w] = 1

    @staticmethod
    def collect(v0, n_own, mine, visited, queue, qn):
        vis = visited.numpy().view(np.uint32)
        q = queue.numpy()
        k = int(qn.item())
        for i in np.nonzero(mine.numpy()[:n_own])[0]:
            v = v0 + int(i)
            b = np.uint32(1) << np.uint32(v & 31)
            if not (vis[v >> 5] & b):
                vis[v >> 5] |= b
                q[k] = v
                k += 1
        qn.fill_(k)


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
        s = giant_scc(fw, bw, g.V, p, ops=CpuOps, device="cpu").numpy().astype(bool)
        q.put((rank, bool(np.array_equal(s, exact == exact[p]))))
    except Exception as e:  # noqa: BLE001
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _worker_scc(rank, world, port, q, kind="planted"):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        g = _graph() if kind == "planted" else _graph_rmat()
        exact = oracle.tarjan(g)
        fw = split_rows(g.fw_beg, g.fw_adj, rank, world)
        bw = split_rows(g.bw_beg, g.bw_adj, rank, world)
        labels = scc(fw, bw, g.V, solve=oracle.tarjan, ops=CpuOps, device="cpu")
        q.put((rank, bool(np.array_equal(labels, exact))))
    except Exception as e:  # noqa: BLE001
        q.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _run_world(world, kind, target=None):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    ps = [ctx.Process(target=target or _worker, args=(r, world, port, q, kind)) for r in range(world)]
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
    # 2048 vertices over 3 ranks: 22, 22 and 20 words of 32 vertices
    res = _run_world(3, "rmat")
    assert res == [(0, True), (1, True), (2, True)], res


def test_split_rows_reassembles_the_csr():
    g = _graph_rmat()
    for world in (1, 2, 3, 5):
        parts = [split_rows(g.fw_beg, g.fw_adj, r, world) for r in range(world)]
        assert [p.v0 for p in parts] == [owned_range(g.V, r, world)[0] for r in range(world)]
        assert all(p.v0 % 32 == 0 for p in parts)  # owned ranges are whole bitmap words
        assert sum(p.n for p in parts) == g.V
        adj = np.concatenate([p.adj for p in parts])
        assert np.array_equal(adj, g.fw_adj)
        deg = np.concatenate([np.diff(p.beg) for p in parts])
        assert np.array_equal(deg, np.diff(g.fw_beg))
    # more ranks than words: empty ranges are valid shards
    tiny_beg, tiny_adj = np.array([0, 1, 2], np.int64), np.array([1, 0], np.int32)
    parts = [split_rows(tiny_beg, tiny_adj, r, 4) for r in range(4)]
    assert [p.n for p in parts] == [2, 0, 0, 0]
    assert np.array_equal(np.concatenate([p.adj for p in parts]), tiny_adj)


def test_allowed_bits_restrict_the_search():
    g = _graph()
    exact = oracle.tarjan(g)
    p = _pivot(g, exact)
    fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
    full = bits_to_map(reach(fw, g.V, [p], None, ops=CpuOps, device="cpu"), g.V)
    scc = (exact == exact[p]).astype(np.uint8)
    words = np.zeros((g.V + 31) // 32, np.uint32)
    idx = np.nonzero(scc)[0]
    np.bitwise_or.at(words, idx >> 5, np.uint32(1) << (idx & 31).astype(np.uint32))
    inside = bits_to_map(reach(fw, g.V, [p], torch.from_numpy(words.view(np.int32)), ops=CpuOps, device="cpu"), g.V)
    assert int(inside.sum()) == int(scc.sum())  # an SCC is closed under reach inside it
    assert int(full.sum()) >= int(inside.sum())


def test_single_rank_matches_oracle():
    g = _graph()
    exact = oracle.tarjan(g)
    p = _pivot(g, exact)
    fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
    bw = split_rows(g.bw_beg, g.bw_adj, 0, 1)
    s = giant_scc(fw, bw, g.V, p, ops=CpuOps, device="cpu").numpy().astype(bool)
    assert np.array_equal(s, exact == exact[p])


def test_seed_set_and_empty_graph():
    g = _graph()
    exact = oracle.tarjan(g)
    fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
    seeds = [0, 1, 2, 3]
    got = bits_to_map(reach(fw, g.V, seeds, None, ops=CpuOps, device="cpu"), g.V).numpy().astype(bool)
    # the union of the seeds' forward sets, by a plain CPU BFS
    want = np.zeros(g.V, bool)
    stack = list(seeds)
    want[seeds] = True
    while stack:
        v = stack.pop()
        for w in g.fw_adj[g.fw_beg[v]:g.fw_beg[v + 1]]:
            if not want[w]:
                want[w] = True
                stack.append(w)
    assert np.array_equal(got, want)
    e = split_rows(np.zeros(41, np.int64), np.zeros(0, np.int32), 0, 1)
    assert int(bits_to_map(reach(e, 40, [7], None, ops=CpuOps, device="cpu"), 40).sum()) == 1
    del exact


def test_sharded_detection_world_size_2():
    """The whole detection over sharded rows: every rank ends with the exact
    labels (trim-1, the giant by the sharded searches, the residual gathered
    and solved; the oracle stands in for the single-GPU engine)."""
    res = _run_world(2, "planted", _worker_scc)
    assert res == [(0, True), (1, True)], res


def test_sharded_detection_world_size_3_uneven_rows():
    res = _run_world(3, "rmat", _worker_scc)
    assert res == [(0, True), (1, True), (2, True)], res


def test_sharded_detection_one_rank_and_trim():
    """One process: labels exact; trim-1 removes exactly vertices that are
    their own SCC; the pivot is active and has the largest degree product."""
    for g in (_graph(), _graph_rmat(), G.toy()):
        exact = oracle.tarjan(g)
        fw = split_rows(g.fw_beg, g.fw_adj, 0, 1)
        bw = split_rows(g.bw_beg, g.bw_adj, 0, 1)
        assert np.array_equal(scc(fw, bw, g.V, solve=oracle.tarjan, ops=CpuOps, device="cpu"), exact)
        active, trimmed = trim1(fw, bw, g.V, rounds=10, device="cpu")
        act = bits_to_map(active, g.V).numpy().astype(bool)
        tr = bits_to_map(trimmed, g.V).numpy().astype(bool)
        assert not (act & tr).any() and (act | tr).all()
        sizes = np.bincount(exact, minlength=g.V)
        assert (sizes[exact[tr]] == 1).all()  # trimmed vertices are singleton SCCs
        p = pivot(fw, bw, g.V, active)
        if act.any():
            prod = np.diff(g.fw_beg).astype(np.int64) * np.diff(g.bw_beg)
            assert act[p] and prod[p] == prod[act].max() and p == np.nonzero(act & (prod == prod[p]))[0][0]

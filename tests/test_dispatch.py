"""Multi-GPU plumbing of the batched/served paths, on CPU: the graph-to-rank
assignment and the world-size-2 gather over gloo, with the oracle standing in
for the per-rank GPU solve (the path has no data-path collective, so this
covers everything the ranks exchange).  A failing rank is made on the host."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from ispan_b200 import graphs as G
from ispan_b200.dispatch import assign_graphs, graph_bytes, run_sharded


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_assign_covers_every_graph_once_and_balances():
    rng = np.random.default_rng(3)
    sizes = [(int(v), int(v * rng.integers(2, 20))) for v in rng.integers(10, 10_000, size=200)]
    for ws in (1, 2, 3, 8):
        a = assign_graphs(sizes, ws)
        flat = sorted(i for share in a for i in share)
        assert flat == list(range(len(sizes)))
        loads = [sum(graph_bytes(*sizes[i]) for i in share) for share in a]
        biggest = max(graph_bytes(*s) for s in sizes)
        assert max(loads) - min(loads) <= biggest  # greedy largest-first bound
        assert a == assign_graphs(sizes, ws)       # every rank computes the same answer


def test_assign_respects_budget():
    sizes = [(1000, 10_000)] * 4
    one = graph_bytes(1000, 10_000)
    assert assign_graphs(sizes, 2, budget_bytes=2 * one) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        assign_graphs(sizes, 2, budget_bytes=one)          # 2 graphs per rank do not fit
    with pytest.raises(ValueError):
        assign_graphs([(10**6, 10**7)], 4, budget_bytes=one)  # one graph alone too big


def _graphs():
    return [G.planted(300 + 50 * i, seed=i, giant_frac=0.3) for i in range(7)] + [G.rmat(8, 8, 2), G.toy()]


def _worker(rank, ws, port, fail_rank, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=10))
    try:
        gs = _graphs()

        def solve(batch):
            if rank == fail_rank:
                raise RuntimeError("injected failure on the host")
            return [oracle.tarjan(g) for g in batch]

        out = run_sharded(gs, [(g.V, g.E) for g in gs], solve)
        if rank == 0:
            ok = all(np.array_equal(o, oracle.tarjan(g)) for o, g in zip(out, gs))
            q.put(("ok", ok))
    except Exception as e:  # noqa: BLE001
        q.put(("err", rank, type(e).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _spawn(fail_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, fail_rank, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(60)
        if p.is_alive():
            p.kill()
    res = []
    while not q.empty():
        res.append(q.get())
    return res


def test_world_size_2_gather_gloo():
    res = _spawn(fail_rank=-1)
    assert ("ok", True) in res, res


def test_world_size_2_failed_rank_is_seen():
    """Rank 1 fails before the gather: it raises locally and rank 0's gather
    ends with an error within the group's timeout instead of hanging."""
    res = _spawn(fail_rank=1)
    errs = {r[1] for r in res if r[0] == "err"}
    assert errs == {0, 1}, res

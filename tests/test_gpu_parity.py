"""GPU parity: the CUDA pipeline, called through the C ABI, against the CPU
oracle (exact Tarjan + serial iSpan restatement) on seeded graphs and on the
golden fixtures taken from the reference.  Integer work: bit-exact labels,
SCC count and size histogram."""
import glob
import os

import numpy as np
import pytest

import oracle
from ispan_b200 import Context, graphs as G

pytestmark = pytest.mark.gpu
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.fixture(scope="module")
def ctx():
    c = Context(1 << 20, 1 << 24)
    yield c
    c.close()


def check(ctx, csr, **kw):
    labels, st = ctx.run_csr(csr, histogram=True, **kw)
    exact = oracle.tarjan(csr)
    bad = np.nonzero(labels != exact)[0]
    assert len(bad) == 0, f"{len(bad)} wrong labels, first {bad[:8]}: gpu {labels[bad[:8]]} exact {exact[bad[:8]]}"
    assert st["scc_count"] == oracle.scc_count(exact)
    assert st["histogram"] == oracle.histogram(exact)
    return st


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_golden(ctx, path):
    z = np.load(path)
    csr = G.CSR(int(z["V"]), int(z["E"]), z["fw_beg"], z["fw_adj"], z["bw_beg"], z["bw_adj"])
    labels, st = ctx.run_csr(csr)
    assert np.array_equal(labels, z["exact"])


@pytest.mark.parametrize("scale,ef,seed", [(8, 16, 1), (12, 16, 2), (16, 16, 1), (16, 16, 3), (14, 4, 5)])
def test_rmat(ctx, scale, ef, seed):
    check(ctx, G.rmat(scale, ef, seed))


def test_rmat_permuted_int64(ctx):
    check(ctx, G.rmat(15, 16, 7, permute=True, offset_dtype=np.int64))


@pytest.mark.parametrize("n,seed,gf", [(2000, 0, 0.3), (20000, 1, 0.3), (20000, 2, 0.0), (50000, 3, 0.5)])
def test_planted(ctx, n, seed, gf):
    check(ctx, G.planted(n, seed, giant_frac=gf))


def test_planted_large_wccs(ctx):
    """Long chains of cycles: WCCs above the shared-memory limit go through the
    colouring rounds."""
    check(ctx, G.planted(60000, 4, giant_frac=0.0, dag_ef=3.0, max_cycle=300))


@pytest.mark.parametrize("seed", range(3))
def test_random_multigraph(ctx, seed):
    check(ctx, G.random_graph(3000, 6000 + 3000 * seed, seed))


def test_edge_cases(ctx):
    check(ctx, G.from_edges(1, np.zeros((0, 2))))
    check(ctx, G.from_edges(100, np.zeros((0, 2))))
    check(ctx, G.from_edges(3, np.array([[0, 0], [1, 1], [2, 2]])))      # self-loops only
    check(ctx, G.from_edges(2, np.array([[0, 1], [1, 0], [0, 1]])))      # duplicate 2-cycle
    cyc = np.array([[i, (i + 1) % 5000] for i in range(5000)])           # one long cycle
    check(ctx, G.from_edges(5000, cyc))
    path = np.array([[i, i + 1] for i in range(4999)])                   # a path: all size-1
    check(ctx, G.from_edges(5000, path))
    check(ctx, G.toy())


def test_malformed_host_input_is_refused(ctx):
    """Host CSRs are checked on the device before any stage runs: offsets
    that fall, do not start at 0 or do not end at E, and ids outside [0, V),
    are refused with ISPAN_ERR_ARG; the context then runs a good graph."""
    from ispan_b200 import IspanError
    good = G.rmat(10, 8, 3)
    bad = []
    fb = good.fw_beg.copy(); fb[5], fb[6] = fb[6], fb[5] - 1            # falling offsets
    bad.append(G.CSR(good.V, good.E, fb, good.fw_adj, good.bw_beg, good.bw_adj))
    bb = good.bw_beg.copy(); bb[-1] -= 1                                 # does not end at E
    bad.append(G.CSR(good.V, good.E, good.fw_beg, good.fw_adj, bb, good.bw_adj))
    fa = good.fw_adj.copy(); fa[7] = good.V                              # id out of range
    bad.append(G.CSR(good.V, good.E, good.fw_beg, fa, good.bw_beg, good.bw_adj))
    for csr in bad:
        with pytest.raises(IspanError) as e:
            ctx.run_csr(csr)
        assert e.value.code == -1  # ISPAN_ERR_ARG
    labels, _ = ctx.run_csr(good)
    assert np.array_equal(labels, oracle.tarjan(good))


def test_device_input_and_repeat(ctx):
    import torch
    csr = G.rmat(14, 16, 9, offset_dtype=np.int64)
    exact = oracle.tarjan(csr)
    d = [torch.from_numpy(a).cuda() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]
    for _ in range(3):  # replays the captured CUDA graph
        labels, st = ctx.run(*d, V=csr.V)
        assert np.array_equal(labels.cpu().numpy(), exact)


def test_batch_union(ctx):
    graphs = [G.rmat(10, 8, s) for s in range(5)] + [G.planted(3000, s) for s in range(5)] + [G.toy()]
    u, vb = G.disjoint_union(graphs)
    labels, st = ctx.run_csr(u, vbase=vb, histogram=True)
    exact = oracle.tarjan(u)
    assert np.array_equal(labels, exact)
    assert st["scc_count"] == oracle.scc_count(exact)
    assert st["histogram"] == oracle.histogram(exact)


def test_stage_times_and_no_graph(ctx):
    """Runs with and without stage times (two cached graphs: with and without
    the event nodes) and direct launches, alternating on one context."""
    csr = G.rmat(13, 16, 4)
    exact = oracle.tarjan(csr)
    for times, use_graph in ((True, True), (False, True), (True, True), (False, False), (True, False), (False, True)):
        labels, st = ctx.run_csr(csr, stage_times=times, use_graph=use_graph)
        assert np.array_equal(labels, exact)
        assert (st["stage_ms"][3] > 0) == times


def test_reference_codes_report(ctx):
    """The reference-convention codes feed the reference's class report; the
    SCC partition they encode (split by induced SCCs) is exact."""
    csr = G.planted(4000, 6)
    labels, st = ctx.run_csr(csr)
    codes = ctx.ref_codes(csr.V)
    assert codes[csr.V] == 0
    assert np.array_equal(oracle.canon_codes(csr, codes), oracle.tarjan(csr))


@pytest.mark.parametrize("tun", [dict(async_v=1, async_e=1, async_deg=1, bfs_ctas_per_sm=1, color_levels=1, color_pivots=1),
                                 dict(async_v=1 << 22, async_e=1 << 24, async_deg=1024, color_levels=100000,
                                      color_pivots=1 << 30),
                                 dict(async_v=4096, async_e=16384, async_deg=4)])
def test_tuning_does_not_change_labels(tun):
    """The autotuner's launch parameters move time between stages only."""
    with Context(1 << 17, 1 << 21) as c:
        c.set_tuning(**tun)
        for g in (G.rmat(14, 16, 9), G.planted(20000, 8, giant_frac=0.3), G.planted(30000, 9, giant_frac=0.0,
                                                                                      dag_ef=3.0, max_cycle=300)):
            for a, b, gm in ((30, 200, 10), (3, 4000, 3), (300, 50, 30)):
                labels, _ = c.run_csr(g, alpha=a, beta=b, gamma=gm)
                assert np.array_equal(labels, oracle.tarjan(g))
        t = c.tuning()
        assert t["async_deg"] == tun["async_deg"]


@pytest.mark.parametrize("pair,pdl", [(1, 0), (-1, 0), (1, -1)])
def test_searches_together_and_in_sequence(pair, pdl):
    """The two giant searches run at the same time (the backward one over all
    active vertices, pivot SCC = F & B) or one after the other (the backward
    one inside F): same labels, same pivot SCC, graph or direct launches,
    plain graphs with 32- and 64-bit offsets and a batch of several graphs."""
    graphs = [G.rmat(15, 16, 2), G.rmat(13, 8, 5, offset_dtype=np.int64), G.planted(40000, 3, giant_frac=0.3),
              G.planted(30000, 4, giant_frac=0.0, dag_ef=3.0, max_cycle=200)]
    with Context(1 << 17, 1 << 21) as c:
        c.set_tuning(pair_searches=pair, pdl=pdl)
        assert c.tuning()["pair_searches"] == pair and c.tuning()["pdl"] == (1 if pdl == 0 else -1)
        for g in graphs:
            exact = oracle.tarjan(g)
            for use_graph, extra in ((True, {}), (False, {}), (True, {"exact_stats": True, "stage_times": True})):
                labels, st = c.run_csr(g, use_graph=use_graph, **extra)
                assert np.array_equal(labels, exact)
                vals, counts = np.unique(exact, return_counts=True)
                assert st["giant_size"] in set(counts.tolist())
                if extra:  # the statistics runs: degree sums of the reached sets, stage times
                    assert st["fw_edges"] >= 0 and st["bw_edges"] >= 0 and st["stage_ms"][3] > 0
        parts = [G.rmat(11, 8, 7), G.planted(3000, 9, giant_frac=0.5), G.rmat(12, 16, 8)]
        u, vb = G.disjoint_union(parts)
        labels, _ = c.run_csr(u, vbase=vb)
        assert np.array_equal(labels, oracle.tarjan(u))


RMAT16 = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "rmat16", "s*.npz")))


@pytest.mark.parametrize("path", RMAT16, ids=[os.path.basename(p)[:-4] for p in RMAT16])
def test_rmat16_against_reference_fixture(ctx, path):
    """The plain-pipeline small workload (R-MAT scale 16, edge factor 16,
    seeds 1-10): GPU labels equal the reference's own OpenMP answer (its raw
    codes from tests/golden/rmat16, canonicalised) and the exact partition."""
    z = np.load(path)
    csr = G.rmat(16, 16, int(z["seed"]))
    assert csr.E == int(z["E"])
    st = check(ctx, csr)
    ref = oracle.canon_codes(csr, z["ref_codes_t16"])
    labels, _ = ctx.run_csr(csr)
    assert np.array_equal(labels, ref)
    assert st["giant_size"] == int((z["ref_codes_t16"][:csr.V] == 1).sum())


@pytest.mark.parametrize("compact", [1, -1])
def test_colouring_on_compact_graph_and_input_graph(compact):
    """More than 65,536 vertices reach the colouring (a DAG of planted cycles
    with no giant SCC), so the compact colouring graph is built when it is on;
    both forms give the exact partition."""
    g = G.planted(150000, 12, giant_frac=0.0, dag_ef=3.0, max_cycle=400)
    with Context(g.V, g.E) as c:
        c.set_tuning(color_compact=compact)
        labels, st = c.run_csr(g, histogram=True)
        assert st["color_rounds"] > 0
        exact = oracle.tarjan(g)
        assert np.array_equal(labels, exact)
        assert st["histogram"] == oracle.histogram(exact)
        assert c.tuning()["color_compact"] == compact


def test_adjacency_at_unaligned_addresses(ctx):
    """Device adjacency arrays that start 4 bytes past a 16-byte boundary (a
    caller's slice): the vectorised loads of the top-down expansion are used
    only at aligned addresses, so the labels are exact either way."""
    import torch
    csr = G.rmat(14, 16, 11, offset_dtype=np.int64)
    exact = oracle.tarjan(csr)
    big = [torch.zeros(len(a) + 1, dtype=torch.int32, device="cuda") for a in (csr.fw_adj, csr.bw_adj)]
    big[0][1:] = torch.from_numpy(csr.fw_adj).cuda()
    big[1][1:] = torch.from_numpy(csr.bw_adj).cuda()
    fa, ba = big[0][1:], big[1][1:]
    assert fa.data_ptr() % 16 == 4 and ba.data_ptr() % 16 == 4
    fb, bb = torch.from_numpy(csr.fw_beg).cuda(), torch.from_numpy(csr.bw_beg).cuda()
    labels, _ = ctx.run(fb, fa, bb, ba, V=csr.V)
    assert np.array_equal(labels.cpu().numpy(), exact)


def _residual_shapes(seed):
    """A giant ring with chords (the pivot's SCC) and, around it, the shapes
    the stages after it handle: peel chains into and out of the ring, sink
    and source 2-cycles, 3-cycles and 3-vertex hubs, a chain of 5-cycles, a
    vertex between two cycles (a size-1 SCC no trim removes), duplicate
    edges and self-loops, in shuffled ids."""
    rng = np.random.default_rng(seed)
    e = []
    ring = list(range(3000))
    e += [(ring[i], ring[(i + 1) % 3000]) for i in range(3000)]
    e += [(int(a), int(b)) for a, b in rng.integers(0, 3000, (6000, 2))]
    nxt = 3000

    def new(k):
        nonlocal nxt
        ids = list(range(nxt, nxt + k))
        nxt += k
        return ids

    for _ in range(20):  # chains out of and into the ring
        c = new(4)
        e += [(int(rng.integers(0, 3000)), c[0]), (c[0], c[1]), (c[1], c[2]), (c[2], c[3])]
        c = new(4)
        e += [(c[0], c[1]), (c[1], c[2]), (c[2], c[3]), (c[3], int(rng.integers(0, 3000)))]
    for _ in range(15):  # sink and source 2-cycles hanging off the ring
        p = new(2)
        e += [(p[0], p[1]), (p[1], p[0]), (int(rng.integers(0, 3000)), p[0])]
        p = new(2)
        e += [(p[0], p[1]), (p[1], p[0]), (p[1], int(rng.integers(0, 3000)))]
    for _ in range(10):  # 3-cycles and hubs
        t = new(3)
        e += [(t[0], t[1]), (t[1], t[2]), (t[2], t[0]), (int(rng.integers(0, 3000)), t[1])]
        h = new(3)
        e += [(h[0], h[1]), (h[1], h[0]), (h[0], h[2]), (h[2], h[0]), (h[2], int(rng.integers(0, 3000)))]
    prev = None
    for _ in range(12):  # a chain of 5-cycles with chords: mice SCCs
        c = new(5)
        e += [(c[i], c[(i + 1) % 5]) for i in range(5)] + [(c[0], c[2])]
        if prev is not None:
            e += [(prev[3], c[1]), (prev[4], c[0])]
        prev = c
    a, mid, b = new(3), new(1), new(3)  # cycle -> vertex -> cycle
    e += [(a[0], a[1]), (a[1], a[2]), (a[2], a[0]), (a[1], mid[0]), (mid[0], b[0]),
          (b[0], b[1]), (b[1], b[2]), (b[2], b[0])]
    d = new(2)  # a duplicated 2-cycle with a self-loop
    e += [(d[0], d[1]), (d[0], d[1]), (d[1], d[0]), (d[1], d[1])]
    perm = rng.permutation(nxt)
    return G.from_edges(nxt, perm[np.asarray(e, np.int64)])


@pytest.mark.parametrize("tiny", [1, 0])
def test_small_residual_in_one_cta(tiny):
    """After the giant SCC only a few hundred vertices remain: with the
    one-CTA path (on request) and with the stage kernels (default), the
    labels, SCC count and size histogram are exact."""
    with Context(1 << 14, 1 << 17) as c:
        c.set_tuning(tiny_residual=tiny)
        assert c.tuning()["tiny_residual"] == (1 if tiny == 1 else -1)
        for seed in (1, 2, 3):
            g = _residual_shapes(seed)
            st = check(c, g)
            assert st["residual"] <= 1024
            assert st["n_trim2"] > 0 and st["n_trim3"] > 0 and st["n_mice_scc"] > 0
            for use_graph in (True, False):
                labels, _ = c.run_csr(g, use_graph=use_graph)
                assert np.array_equal(labels, oracle.tarjan(g))
        for seed in range(6):  # random graphs with self-loops and duplicates
            check(c, G.random_graph(3000, 9000 + 1000 * seed, seed))
        check(c, G.rmat(12, 8, 4))


def test_small_residual_counts_match_stage_kernels():
    """The one-CTA path records the stage kernels' classification: peeled,
    trim-2, trim-3 and mice counts equal with the path on and off."""
    keys = ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3", "n_mice_scc", "n_mice_vertices")
    got = {}
    for tiny in (1, 0):
        with Context(1 << 14, 1 << 17) as c:
            c.set_tuning(tiny_residual=tiny)
            _, st = c.run_csr(_residual_shapes(4))
            got[tiny] = {k: st[k] for k in keys}
    assert got[1] == got[0]

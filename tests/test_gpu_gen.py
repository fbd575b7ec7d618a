"""GPU generators: well-formed CSR, the intended SCC structure, and GPU
pipeline labels equal to the oracle on scaled-down versions of the benchmark
graphs."""
import numpy as np
import pytest

import oracle
from ispan_b200 import Context, gen, graphs as G

pytestmark = pytest.mark.gpu


def exact_check(csr, **kw):
    with Context(csr.V, csr.E) as ctx:
        labels, st = ctx.run_csr(csr, histogram=True, **kw)
    exact = oracle.tarjan(csr)
    assert np.array_equal(labels, exact)
    assert st["histogram"] == oracle.histogram(exact)
    return exact, st


def test_rmat_matches_numpy_shape():
    g = gen.rmat(12, 16, 3)
    csr = g.to_host(np.int32)
    G.validate(csr)
    assert csr.V == 4096 and 0.8 * 16 * 4096 < csr.E <= 16 * 4096
    exact_check(csr)


def test_social_small_structure_and_parity():
    g = gen.social(seed=2, scale=0.005)
    csr = g.to_host(np.int64)
    G.validate(csr)
    exact, st = exact_check(csr)
    hist = oracle.histogram(exact)
    big = max(hist)
    assert abs(big / csr.V - 0.80) < 0.02          # giant SCC ~80 % of vertices
    assert hist.get(2, 0) >= 0.9 * int(80112 * 0.005)  # planted 2-cycles survive as SCCs
    lab0 = exact[0]
    assert (exact == lab0).sum() == big             # vertex 0 is in the giant SCC


def test_web_small_parity():
    g = gen.web(seed=3, scale=0.0005)
    csr = g.to_host(np.int64)
    G.validate(csr)
    exact, st = exact_check(csr)
    hist = oracle.histogram(exact)
    assert max(hist) > 0.3 * csr.V


def test_batch_small_parity():
    g = gen.batch(nseg=24, vmin=100, vmax=5000, ef_min=4, ef_max=12, max_cycle=40, seed=5)
    csr = g.to_host(np.int32)
    G.validate(csr)
    with Context(csr.V, csr.E) as ctx:
        labels, st = ctx.run_csr(csr, vbase=g.vbase, histogram=True)
    exact = oracle.tarjan(csr)
    assert np.array_equal(labels, exact)
    # labels never cross graph boundaries
    seg = np.searchsorted(g.vbase, np.arange(csr.V), side="right") - 1
    assert np.array_equal(seg, np.searchsorted(g.vbase, labels, side="right") - 1)


def test_social_medium_repeated_runs_exact():
    """Repeated runs on one context (graph replay, state left by the previous
    run) stay exact on a 2 %-scale social graph."""
    g = gen.social(seed=4, scale=0.02)
    csr = g.to_host(np.int64)
    exact = oracle.tarjan(csr)
    with Context(csr.V, csr.E) as ctx:
        for use_graph in (False, True, True, True):
            labels, st = ctx.run_csr(csr, use_graph=use_graph)
            assert np.array_equal(labels, exact)


@pytest.mark.parametrize("kind,scale,seed", [("social", 0.005, 3), ("web", 0.004, 2)])
def test_planted_partition_is_exact(kind, scale, seed):
    """The generators' planted partition equals the exact SCC partition
    (pins it as a full-size reference for the tests below)."""
    g = getattr(gen, kind)(seed=seed, scale=scale)
    planted = g.planted_labels().cpu().numpy()
    exact = oracle.tarjan(g.to_host(np.int64))
    assert np.array_equal(planted, exact)


@pytest.mark.parametrize("kind,scale", [("social", 1.0), ("web", 0.2)])
def test_large_graph_labels_equal_planted_partition(kind, scale):
    """Full-size social graph (41.6 M vertices, 1.47 B edges) and a 140 M-vertex
    web graph: every label equals the planted partition's, compared on the
    device."""
    import torch
    g = getattr(gen, kind)(seed=1, scale=scale)
    with Context(g.V, g.E) as ctx:
        lab = torch.empty(g.V, dtype=torch.int32, device="cuda")
        fb, fa, bb, ba = g.ptrs
        _, st = ctx.run_raw(g.V, g.E, fb, fa, bb, ba, 8, lab)
        planted = g.planted_labels()
        assert int((lab != planted).sum()) == 0
        n_scc = int((planted == torch.arange(g.V, dtype=torch.int32, device="cuda")).sum())
        assert st["scc_count"] == n_scc
    g.free()


@pytest.mark.parametrize("on_device", [False, True])
def test_csr_from_edge_list(on_device):
    """GPU CSR construction from an edge list equals the host construction of
    the deduplicated list (both directions, adjacency sorted); the SCC labels
    of the raw list (duplicates and self-loops kept) are the same."""
    import torch
    rng = np.random.default_rng(11)
    V, m = 3000, 20000
    e = rng.integers(0, V, size=(m, 2))
    e = np.concatenate([e, e[:500], np.stack([np.arange(50), np.arange(50)], 1)])  # duplicates, self-loops
    src, dst = e[:, 0].astype(np.int32), e[:, 1].astype(np.int32)
    if on_device:
        g = gen.from_edges(V, torch.from_numpy(src).cuda(), torch.from_numpy(dst).cuda())
    else:
        g = gen.from_edges(V, src, dst)
    got = g.to_host(np.int64)
    want = G.from_edges(V, G.dedupe_edges(e), offset_dtype=np.int64)
    for k in ("fw_beg", "fw_adj", "bw_beg", "bw_adj"):
        assert np.array_equal(getattr(got, k), getattr(want, k)), k
    assert np.array_equal(oracle.tarjan(got), oracle.tarjan(G.from_edges(V, e)))
    g.free()
    with pytest.raises(RuntimeError):
        gen.from_edges(10, np.array([0, 11], np.int32), np.array([1, 2], np.int32))

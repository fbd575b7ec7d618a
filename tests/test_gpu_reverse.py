"""Forward-only input: the reverse CSR built on the device (bw_beg and bw_adj
both NULL in ispan_csr), for host and device graphs.  Labels, SCC count and
size histogram against the oracle; malformed forward CSRs are refused with
ISPAN_ERR_ARG and leave the context usable."""
import glob
import os

import numpy as np
import pytest

import oracle
from ispan_b200 import Context, IspanError, graphs as G

pytestmark = pytest.mark.gpu
GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.fixture(scope="module")
def ctx():
    c = Context(1 << 20, 1 << 24)
    yield c
    c.close()


def check_fw_only(ctx, csr, device=False, atomic=False):
    exact = oracle.tarjan(csr)
    if device:
        import torch
        fb, fa = (torch.from_numpy(a).cuda() for a in (csr.fw_beg, csr.fw_adj))
        labels, st = ctx.run(fb, fa, V=csr.V, histogram=True, reverse_atomic=atomic)
        labels = labels.cpu().numpy()
    else:
        labels, st = ctx.run(csr.fw_beg, csr.fw_adj, V=csr.V, histogram=True, reverse_atomic=atomic)
    bad = np.nonzero(labels != exact)[0]
    assert len(bad) == 0, f"{len(bad)} wrong labels, first {bad[:8]}"
    assert st["scc_count"] == oracle.scc_count(exact)
    assert st["histogram"] == oracle.histogram(exact)


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_golden_forward_only(ctx, path):
    z = np.load(path)
    labels, _ = ctx.run(z["fw_beg"], z["fw_adj"], V=int(z["V"]))
    assert np.array_equal(labels, z["exact"])


@pytest.mark.parametrize("atomic", [False, True], ids=["sorted", "atomic"])
@pytest.mark.parametrize("device", [False, True], ids=["host", "device"])
@pytest.mark.parametrize("make", [
    lambda: G.rmat(14, 16, 2),
    lambda: G.rmat(15, 16, 7, permute=True, offset_dtype=np.int64),
    lambda: G.planted(50000, 3, giant_frac=0.5),
    lambda: G.planted(60000, 4, giant_frac=0.0, dag_ef=3.0, max_cycle=300),
    lambda: G.toy(),
], ids=["rmat14", "rmat15_int64", "planted", "planted_large_wccs", "toy"])
def test_forward_only(ctx, make, device, atomic):
    check_fw_only(ctx, make(), device, atomic)


@pytest.mark.parametrize("atomic", [False, True], ids=["sorted", "atomic"])
def test_forward_only_several_chunks(ctx, atomic):
    """More than 2^22 edges: the forward adjacency is copied in chunks, each
    counted as it lands."""
    csr = G.rmat(19, 16, 5, offset_dtype=np.int64)
    assert csr.E > 1 << 22
    check_fw_only(ctx, csr, atomic=atomic)


@pytest.mark.parametrize("atomic", [False, True], ids=["sorted", "atomic"])
def test_forward_only_self_loops_duplicates_and_empty(ctx, atomic):
    """Self-loops, duplicate edges, isolated vertices, no edges at all."""
    edges = np.array([[0, 0], [0, 1], [1, 0], [1, 0], [2, 2], [3, 4], [4, 5], [5, 3], [5, 3], [6, 7]], np.int64)
    check_fw_only(ctx, G.from_edges(9, edges), atomic=atomic)
    check_fw_only(ctx, G.from_edges(5, np.zeros((0, 2), np.int64)), atomic=atomic)
    check_fw_only(ctx, G.from_edges(1, np.zeros((0, 2), np.int64)), atomic=atomic)


@pytest.mark.parametrize("atomic", [False, True], ids=["sorted", "atomic"])
def test_forward_only_hub_lists(ctx, atomic):
    """Lists of 32 edges and more are placed by a whole warp: a star in both
    directions around hub 0 plus a ring (one SCC of everything)."""
    n = 5000
    ring = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
    star = np.concatenate([np.stack([np.zeros(n - 1, np.int64), np.arange(1, n)], 1),
                           np.stack([np.arange(1, n), np.zeros(n - 1, np.int64)], 1)])
    check_fw_only(ctx, G.from_edges(n, np.concatenate([ring, star]).astype(np.int64)), atomic=atomic)


def test_derived_reverse_gives_the_same_run(ctx):
    """A run on the derived reverse CSR and a run on the given one agree in
    their stage statistics as well as their labels (the reverse lists hold
    the same ids, in another order)."""
    csr = G.rmat(16, 16, 4)
    a_lab, a = ctx.run(csr.fw_beg, csr.fw_adj, V=csr.V, exact_stats=True)
    b_lab, b = ctx.run_csr(csr, exact_stats=True)
    assert np.array_equal(a_lab, b_lab)
    for k in ("scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3", "fw_size", "residual", "fw_edges",
              "bw_edges"):
        assert a[k] == b[k], k


@pytest.mark.parametrize("atomic", [False, True], ids=["sorted", "atomic"])
def test_forward_only_malformed_is_refused(ctx, atomic):
    good = G.rmat(10, 8, 3)
    bad = []
    fb = good.fw_beg.copy(); fb[5], fb[6] = fb[6], fb[5] - 1   # falling offsets
    bad.append((fb, good.fw_adj))
    fb = good.fw_beg.copy(); fb[-1] -= 1                      # does not end at E
    bad.append((fb, good.fw_adj))
    fb = good.fw_beg.copy(); fb[0] = 1                        # does not start at 0
    bad.append((fb, good.fw_adj))
    fa = good.fw_adj.copy(); fa[7] = good.V                   # id out of range
    bad.append((good.fw_beg, fa))
    fa = good.fw_adj.copy(); fa[3] = -5                       # negative id
    bad.append((good.fw_beg, fa))
    for fb, fa in bad:
        with pytest.raises(IspanError) as e:
            ctx.run(fb, fa, V=good.V, reverse_atomic=atomic)
        assert e.value.code == -1  # ISPAN_ERR_ARG
    check_fw_only(ctx, good, atomic=atomic)


def test_one_reverse_array_is_an_error(ctx):
    g = G.rmat(8, 8, 1)
    with pytest.raises(ValueError):
        ctx.run(g.fw_beg, g.fw_adj, g.bw_beg, None, V=g.V)

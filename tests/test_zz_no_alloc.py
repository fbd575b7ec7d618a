"""The allocation-free entry point, ispan_scc_small_noalloc.

Some callers cannot allocate device memory: code running under another
framework's memory manager (which owns the device memory), paths that cannot
take cudaMalloc's implicit synchronisation, or work issued while a stream is
being captured.  For them the library offers one entry point whose scratch is
a fixed array compiled into the library.  These tests call it through the C
ABI on device-resident graphs, on two calls in a row (the second reuses the
scratch the first left behind), and check its labels against the exact
partition of the CPU oracle (Tarjan) and against the regular entry point,
ispan_scc_run.  The labels are integers: they must be identical.  The
capacity edge is covered too: exactly ISPAN_NOALLOC_MAX_V vertices, as one
cycle and as one path, which drive the kernel's explicit stacks to full depth.
This file is collected last on purpose, so a run that stops at the first
failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from ispan_b200 import Context, _lib, graphs as G

pytestmark = pytest.mark.gpu


def _dev(csr):
    import torch
    return [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]


def _csr_struct(V, E, fb, fa, bb, ba):
    return _lib.Csr(V, E, fb.data_ptr(), bb.data_ptr(), fa.data_ptr(), ba.data_ptr(), fb.element_size(), 1)


def _noalloc(g, V):
    import torch
    out = torch.full((V,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.lib().ispan_scc_small_noalloc(C.byref(g), C.c_void_p(out.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _check_twice(csr):
    d = _dev(csr)
    exact = oracle.tarjan(csr)
    with Context(csr.V, csr.E) as ctx:
        regular, _ = ctx.run(*d, V=csr.V)
        regular = regular.cpu().numpy().copy()
    assert np.array_equal(regular, exact)
    g = _csr_struct(csr.V, csr.E, *d)
    for call in range(2):
        rc, out = _noalloc(g, csr.V)
        assert rc == 0, f"call {call}: {rc}"
        assert np.array_equal(out, exact), f"call {call} differs from the oracle"
        assert np.array_equal(out, regular), f"call {call} differs from ispan_scc_run"


@pytest.mark.parametrize("offsets", [np.int32, np.int64])
def test_noalloc_matches_oracle_and_regular_entry_point(offsets):
    _check_twice(G.planted(30000, 11, giant_frac=0.25, offset_dtype=offsets))


def test_noalloc_full_capacity_cycle_and_path():
    V = _lib.NOALLOC_MAX_V
    ring = np.stack([np.arange(V), (np.arange(V) + 1) % V], 1)
    _check_twice(G.from_edges(V, ring))             # one SCC; the DFS goes V deep
    path = np.stack([np.arange(V - 1), np.arange(1, V)], 1)
    _check_twice(G.from_edges(V, path))             # V singletons, V deep as well


def test_noalloc_rejects_graphs_above_its_scratch():
    import torch
    V = _lib.NOALLOC_MAX_V + 1
    fb = torch.zeros(V + 1, dtype=torch.int32, device="cuda")
    fa = torch.zeros(1, dtype=torch.int32, device="cuda")
    g = _csr_struct(V, 0, fb, fa, fb, fa)
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    rc = _lib.lib().ispan_scc_small_noalloc(C.byref(g), C.c_void_p(out.data_ptr()), None)
    assert rc == -7  # ISPAN_ERR_CAPACITY


def test_noalloc_malformed_graph_gets_minus_one_labels():
    """An adjacency id outside [0, V) (offsets still well formed, so every
    read stays inside the arrays) is caught by the kernel's input check: every
    label is -1, no fault, and the next call on a good graph is exact."""
    csr = G.planted(2000, 3, giant_frac=0.3)
    d = _dev(csr)
    bad_adj = d[1].clone()
    bad_adj[bad_adj.numel() // 2] = csr.V + 5
    rc, out = _noalloc(_csr_struct(csr.V, csr.E, d[0], bad_adj, d[2], d[3]), csr.V)
    assert rc == 0 and (out == -1).all()
    bad_beg = d[0].clone()
    bad_beg[csr.V] = csr.E - 1  # offsets must end at E
    rc, out = _noalloc(_csr_struct(csr.V, csr.E, bad_beg, d[1], d[2], d[3]), csr.V)
    assert rc == 0 and (out == -1).all()
    rc, out = _noalloc(_csr_struct(csr.V, csr.E, *d), csr.V)
    assert rc == 0 and np.array_equal(out, oracle.tarjan(csr))

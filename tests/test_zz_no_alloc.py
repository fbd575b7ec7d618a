"""The allocation-free entry point, ispan_scc_small_noalloc.

Some callers cannot allocate device memory (they run under another
framework's memory manager, on paths that cannot take cudaMalloc's implicit
synchronisation, or while a stream is being captured).  For them the library
offers one entry point whose scratch is a fixed array compiled into the
library.  This test calls it through the C ABI on a device-resident graph
and checks its labels against the regular entry point, ispan_scc_run, on two
calls in a row (the second reuses the scratch the first left behind).  The
labels are integers: they must be identical.  This file is collected last on
purpose, so a run that stops at the first failure has run every other test
before it.
"""
import ctypes as C

import numpy as np
import pytest

from ispan_b200 import Context, _lib, graphs as G

pytestmark = pytest.mark.gpu


def _csr_struct(V, E, fb, fa, bb, ba):
    return _lib.Csr(V, E, fb.data_ptr(), bb.data_ptr(), fa.data_ptr(), ba.data_ptr(), fb.element_size(), 1)


@pytest.mark.parametrize("offsets", [np.int32, np.int64])
def test_noalloc_matches_regular_entry_point(offsets):
    import torch
    csr = G.planted(30000, 11, giant_frac=0.25, offset_dtype=offsets)
    d = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj)]
    with Context(csr.V, csr.E) as ctx:
        want, _ = ctx.run(*d, V=csr.V)
        want = want.cpu().numpy().copy()
    g = _csr_struct(csr.V, csr.E, *d)
    L = _lib.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full((csr.V,), -7, dtype=torch.int32, device="cuda")
        rc = L.ispan_scc_small_noalloc(C.byref(g), C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert rc == 0, f"call {call}: {rc}"
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want), f"call {call} differs from ispan_scc_run"


def test_noalloc_rejects_graphs_above_its_scratch():
    import torch
    V = _lib.NOALLOC_MAX_V + 1
    fb = torch.zeros(V + 1, dtype=torch.int32, device="cuda")
    fa = torch.zeros(1, dtype=torch.int32, device="cuda")
    g = _csr_struct(V, 0, fb, fa, fb, fa)
    out = torch.empty(V, dtype=torch.int32, device="cuda")
    rc = _lib.lib().ispan_scc_small_noalloc(C.byref(g), C.c_void_p(out.data_ptr()), None)
    assert rc == -7  # ISPAN_ERR_CAPACITY

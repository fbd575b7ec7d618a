"""Failure detection on the GPU without a fault: the persistent stages'
bounded grid barrier, run with a CTA that never arrives, gives up after its
limit, reports ISPAN_ERR_TIMEOUT, and the context stays usable."""
import time

import numpy as np
import pytest

import oracle
from ispan_b200 import Context, _lib, graphs as G

pytestmark = pytest.mark.gpu


def test_barrier_wait_times_out_and_context_survives():
    g = G.planted(3000, 4, giant_frac=0.3)
    with Context(g.V, g.E) as ctx:
        before, _ = ctx.run_csr(g)
        t0 = time.monotonic()
        rc = _lib.lib().ispan_debug_barrier_timeout(ctx._h, 200_000)  # 0.2 s
        dt = time.monotonic() - t0
        assert rc == -4  # ISPAN_ERR_TIMEOUT
        assert 0.15 < dt < 10.0
        after, _ = ctx.run_csr(g)  # the same context runs a graph afterwards
        assert np.array_equal(before, after)
        assert np.array_equal(after, oracle.tarjan(g))


def test_barrier_probe_rejects_bad_limits():
    with Context(16, 16) as ctx:
        assert _lib.lib().ispan_debug_barrier_timeout(ctx._h, 0) == -1
        assert _lib.lib().ispan_debug_barrier_timeout(ctx._h, 11_000_000) == -1

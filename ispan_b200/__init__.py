"""ispan_b200 -- strongly connected components on one B200 (sm_100a).

A drop-in for iSpan's detection call.  The host-side mirror of the
reference's interface lives here, with the reference's names, argument
meaning and error behaviour replaced by exceptions:

* :class:`graph` / :func:`graph_load`   -- src/graph.h:9-31, src/load_print.cpp:6-22
* :func:`scc_detection`                 -- src/scc_common.h:15-23 (src/scc_core.cpp:27)
* :func:`get_scc_result`                -- src/load_print.cpp:24-60 (class report)
* :func:`print_time_result`             -- src/load_print.cpp:62-92

plus :class:`Context`, the direct interface to the CUDA engine (device or
host CSR, canonical labels, statistics, batched graphs).  All computation
runs in libispan_b200.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import IspanError, check
from .graphs import CSR, read_bin

__all__ = ["Context", "Server", "condensation", "graph", "graph_load", "scc_detection", "get_scc_result", "print_time_result",
           "IspanError", "CSR", "scc"]

REFERENCE_DEFAULTS = dict(alpha=30, beta=200, gamma=10, theta=0.1)  # src/bash_one.sh:4


def _ptr(a) -> int:
    """Data pointer of a numpy array or a torch tensor (0 for None)."""
    if a is None:
        return 0
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


class Context:
    """Device scratch for graphs up to ``max_V`` vertices and ``max_E`` edges
    on one GPU.  Reuse it across runs: the stage sequence is captured into a
    CUDA graph on the first run of a given shape and replayed."""

    def __init__(self, max_V: int, max_E: int, device: int = 0):
        L = _lib.lib()
        h = C.c_void_p()
        check(L.ispan_ctx_create(device, int(max_V), int(max_E), C.byref(h)), "ispan_ctx_create")
        self._h = h
        self.max_V, self.max_E, self.device = int(max_V), int(max_E), device
        self._keep = None

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().ispan_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream) -> None:
        """Run on a caller's CUDA stream (torch.cuda.Stream or raw handle)."""
        handle = getattr(stream, "cuda_stream", stream)
        check(_lib.lib().ispan_ctx_set_stream(self._h, C.c_void_p(int(handle))), "set_stream")

    @staticmethod
    def _csr_struct(V, E, fw_beg, fw_adj, bw_beg, bw_adj, on_device: bool) -> _lib.Csr:
        ob = fw_beg.element_size() if hasattr(fw_beg, "element_size") else fw_beg.dtype.itemsize
        return _lib.Csr(int(V), int(E), _ptr(fw_beg), _ptr(bw_beg), _ptr(fw_adj), _ptr(bw_adj), ob,
                        1 if on_device else 0)

    def set_tuning(self, async_v=0, async_e=0, async_deg=0, bfs_ctas_per_sm=0, color_levels=0,
                   color_pivots=0, color_compact=0, pair_searches=0, tiny_residual=0, pdl=0) -> None:
        """Launch tunables (zero = default); see ispan_b200.autotune."""
        t = _lib.Tuning(int(async_v), int(async_e), int(async_deg), int(bfs_ctas_per_sm), int(color_levels),
                        int(color_pivots), int(color_compact), int(pair_searches), int(tiny_residual), int(pdl))
        check(_lib.lib().ispan_ctx_set_tuning(self._h, C.byref(t)), "ispan_ctx_set_tuning")

    def tuning(self) -> dict:
        t = _lib.Tuning()
        check(_lib.lib().ispan_ctx_get_tuning(self._h, C.byref(t)), "ispan_ctx_get_tuning")
        return t.as_dict()

    def run(self, fw_beg, fw_adj, bw_beg=None, bw_adj=None, V: int | None = None, labels_out=None,
            vbase=None, alpha=30, beta=200, gamma=10, theta=0.1, stage_times=False, use_graph=True,
            histogram=False, exact_stats=False, validate=False, reverse_atomic=False):
        """Detect SCCs.  Arrays are numpy (host) or torch CUDA tensors (device);
        offsets int32 or int64, ids int32.  Returns (labels, stats): labels[V]
        int32 canonical min-id labels, a numpy array for host input or the
        given/new CUDA tensor for device input.  ``vbase`` (numpy int64,
        nseg+1 entries) runs a disjoint union of graphs as a batch.  With
        ``bw_beg`` and ``bw_adj`` both None, only the forward CSR is given
        (and, for host input, copied): the reverse is built on the device,
        by a sort or, with ``reverse_atomic``, by atomics (no scratch)."""
        if (bw_beg is None) != (bw_adj is None):
            raise ValueError("give both reverse arrays or neither")
        on_dev = hasattr(fw_beg, "is_cuda") and fw_beg.is_cuda
        if V is None:
            V = (fw_beg.numel() if hasattr(fw_beg, "numel") else len(fw_beg)) - 1
        E = fw_adj.numel() if hasattr(fw_adj, "numel") else len(fw_adj)
        for a in (fw_beg, fw_adj, bw_beg, bw_adj):
            if hasattr(a, "is_contiguous") and not a.is_contiguous():
                raise ValueError("arrays must be contiguous")
        g = self._csr_struct(V, E, fw_beg, fw_adj, bw_beg, bw_adj, on_dev)
        flags = 0
        if stage_times:
            flags |= _lib.F_STAGE_TIMES
        if not use_graph:
            flags |= _lib.F_NO_GRAPH
        if exact_stats:
            flags |= _lib.F_EXACT_STATS
        if validate:
            flags |= _lib.F_VALIDATE
        if reverse_atomic:
            flags |= _lib.F_REVERSE_ATOMIC
        if on_dev:
            import torch
            if labels_out is None:
                labels_out = torch.empty(max(V, 1), dtype=torch.int32, device=fw_beg.device)
            flags |= _lib.F_LABELS_ON_DEVICE
        else:
            if labels_out is None:
                labels_out = np.empty(max(V, 1), np.int32)
        p = _lib.Params(alpha, beta, gamma, theta, flags)
        st = _lib.Stats()
        hs = hc = None
        if histogram:
            cap = 1 << 17
            hs = np.zeros(cap, np.int64)
            hc = np.zeros(cap, np.int64)
            st.hist_size, st.hist_count, st.hist_cap = hs.ctypes.data, hc.ctypes.data, cap
        L = _lib.lib()
        if vbase is None:
            rc = L.ispan_scc_run(self._h, C.byref(g), C.byref(p), C.c_void_p(_ptr(labels_out)), C.byref(st))
        else:
            vb = np.ascontiguousarray(vbase, np.int64)
            rc = L.ispan_scc_run_batch(self._h, C.byref(g), len(vb) - 1, vb.ctypes.data, C.byref(p),
                                       C.c_void_p(_ptr(labels_out)), C.byref(st))
        check(rc, "ispan_scc_run")
        stats = st.as_dict()
        if histogram:
            n = min(st.hist_n, st.hist_cap)
            stats["histogram"] = {int(s): int(c) for s, c in zip(hs[:n], hc[:n])}
        return labels_out[:V], stats

    def run_raw(self, V, E, fw_beg, fw_adj, bw_beg, bw_adj, offset_bytes, labels_out, vbase=None,
                alpha=30, beta=200, gamma=10, theta=0.1, stage_times=False, exact_stats=False):
        """Run on raw device pointers (e.g. a generator's arrays, no copy);
        labels_out is a CUDA tensor of V int32."""
        g = _lib.Csr(int(V), int(E), int(fw_beg), int(bw_beg), int(fw_adj), int(bw_adj), int(offset_bytes), 1)
        flags = _lib.F_LABELS_ON_DEVICE | (_lib.F_STAGE_TIMES if stage_times else 0) | \
            (_lib.F_EXACT_STATS if exact_stats else 0)
        p = _lib.Params(alpha, beta, gamma, theta, flags)
        st = _lib.Stats()
        L = _lib.lib()
        if vbase is None:
            rc = L.ispan_scc_run(self._h, C.byref(g), C.byref(p), C.c_void_p(_ptr(labels_out)), C.byref(st))
        else:
            vb = np.ascontiguousarray(vbase, np.int64)
            rc = L.ispan_scc_run_batch(self._h, C.byref(g), len(vb) - 1, vb.ctypes.data, C.byref(p),
                                       C.c_void_p(_ptr(labels_out)), C.byref(st))
        check(rc, "ispan_scc_run")
        return labels_out, st.as_dict()

    def run_graphs(self, graphs, labels_out=None, alpha=30, beta=200, gamma=10, theta=0.1,
                   use_graph=False):
        """Many independent graphs in one set of stage launches.  ``graphs`` is
        a list of (fw_beg, fw_adj, bw_beg, bw_adj) -- numpy (host) or torch
        CUDA tensors (device), each graph on its own side.  Returns one label
        array per graph (local min ids; host graphs get numpy arrays, device
        graphs CUDA tensors unless ``labels_out`` gives the buffers) and the
        batch statistics."""
        n = len(graphs)
        arr = (_lib.Csr * n)()
        outs = []
        for i, (fb, fa, bb, ba) in enumerate(graphs):
            on_dev = hasattr(fb, "is_cuda") and fb.is_cuda
            V = (fb.numel() if hasattr(fb, "numel") else len(fb)) - 1
            E = fa.numel() if hasattr(fa, "numel") else len(fa)
            arr[i] = self._csr_struct(V, E, fb, fa, bb, ba, on_dev)
            if labels_out is not None:
                outs.append(labels_out[i])
            elif on_dev:
                import torch
                outs.append(torch.empty(max(V, 1), dtype=torch.int32, device=fb.device))
            else:
                outs.append(np.empty(max(V, 1), np.int32))
        ptrs = (C.c_void_p * n)(*[_ptr(o) for o in outs])
        p = _lib.Params(alpha, beta, gamma, theta, 0 if use_graph else _lib.F_NO_GRAPH)
        st = _lib.Stats()
        check(_lib.lib().ispan_scc_run_graphs(self._h, arr, n, ptrs, C.byref(p), C.byref(st)),
              "ispan_scc_run_graphs")
        return [o[:arr[i].V] for i, o in enumerate(outs)], st.as_dict()

    def run_csr(self, csr: CSR, **kw):
        return self.run(csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj, V=csr.V, **kw)

    def trace(self):
        """Per-level records of the last run: FW and BW searches (mode, reached,
        frontier_edges, t_ns), the large-WCC rounds (round, left, pivots, t_ns)
        and, for a run with exact_stats, each round's relaxation counts (pops,
        edges, queued, pool-wait ns)."""
        t = np.zeros(4 * 256 * 4, np.int64)
        check(_lib.lib().ispan_debug_trace(self._h, t.ctypes.data, len(t)), "ispan_debug_trace")
        t = t.reshape(4, 256, 4)
        out = []
        for d in range(3):
            rows = [tuple(int(x) for x in r) for r in t[d] if r[3] != 0]
            out.append(rows)
        # with exact_stats: per colouring round, the forward relaxation's pops,
        # edges checked, vertices queued and pool-wait ns summed over warps
        out.append([tuple(int(x) for x in r) for r in t[3][:len(out[2])]])
        return out

    def ref_codes(self, V: int) -> np.ndarray:
        """scc_id codes of the last run in the reference's convention, [V+1]."""
        out = np.empty(V + 1, np.int32)
        check(_lib.lib().ispan_ref_codes(self._h, out.ctypes.data), "ispan_ref_codes")
        return out


class Server:
    """Served form (ispan_server_* of include/ispan_b200.h): submit graphs one
    at a time; ``n_slots`` lanes (default 4) take the queued requests as they
    free up and run their batches (one disjoint union each) concurrently on
    the GPU, each batch's memory taken from the ``hbm_budget_bytes`` budget
    while it runs.  Each request's arrays and label buffer must stay alive
    until the request is reported done (the object keeps references)."""

    def __init__(self, device=0, hbm_budget_bytes=0, max_batch_graphs=0, max_batch_V=0, max_batch_E=0,
                 max_wait_us=0, max_pending=0, alpha=30, beta=200, gamma=10, theta=0.1, use_graph=False,
                 n_slots=0):
        cfg = _lib.ServerConfig(device, max_batch_graphs, n_slots, 0, hbm_budget_bytes, max_batch_V, max_batch_E,
                                max_wait_us, max_pending,
                                _lib.Params(alpha, beta, gamma, theta, 0 if use_graph else _lib.F_NO_GRAPH))
        h = C.c_void_p()
        check(_lib.lib().ispan_server_create(C.byref(cfg), C.byref(h)), "ispan_server_create")
        self._h = h
        self._keep: dict = {}
        self._done: dict = {}  # finished requests seen by peek()

    def limits(self):
        v, e, n = C.c_int64(), C.c_int64(), C.c_int32()
        check(_lib.lib().ispan_server_limits(self._h, C.byref(v), C.byref(e), C.byref(n)), "limits")
        return v.value, e.value, n.value

    def submit(self, fw_beg, fw_adj, bw_beg, bw_adj, labels_out) -> int:
        on_dev = hasattr(fw_beg, "is_cuda") and fw_beg.is_cuda
        V = (fw_beg.numel() if hasattr(fw_beg, "numel") else len(fw_beg)) - 1
        E = fw_adj.numel() if hasattr(fw_adj, "numel") else len(fw_adj)
        g = Context._csr_struct(V, E, fw_beg, fw_adj, bw_beg, bw_adj, on_dev)
        t = C.c_int64()
        check(_lib.lib().ispan_server_submit(self._h, C.byref(g), C.c_void_p(_ptr(labels_out)), C.byref(t)),
              "ispan_server_submit")
        self._keep[t.value] = (fw_beg, fw_adj, bw_beg, bw_adj, labels_out)
        return t.value

    def poll(self, ticket: int):
        """None while queued or running, else the request's info dict."""
        if ticket in self._done:
            return self._finish(ticket, *self._done.pop(ticket))
        info = _lib.RequestInfo()
        rc = _lib.lib().ispan_server_poll(self._h, ticket, C.byref(info))
        if rc == 0:
            return None
        return self._finish(ticket, rc, info.as_dict())

    def peek(self, ticket: int) -> dict:
        """The request's info without consuming it: status 0 while queued or
        running (t_start_ns is set once its batch is admitted)."""
        if ticket in self._done:
            return dict(self._done[ticket][1])
        info = _lib.RequestInfo()
        rc = _lib.lib().ispan_server_poll(self._h, ticket, C.byref(info))
        d = info.as_dict()
        if rc != 0:  # finished: the library reported it once; keep it for poll/wait
            self._done[ticket] = (rc, d)
        return dict(d)

    def wait(self, ticket: int, timeout_s: float | None = None):
        if ticket in self._done:
            return self._finish(ticket, *self._done.pop(ticket))
        info = _lib.RequestInfo()
        us = -1 if timeout_s is None else int(timeout_s * 1e6)
        rc = _lib.lib().ispan_server_wait(self._h, ticket, us, C.byref(info))
        if rc == 0:
            return None
        return self._finish(ticket, rc, info.as_dict())

    def _finish(self, ticket, rc, info):
        self._keep.pop(ticket, None)
        check(rc if rc < 0 else 0, "request %d" % ticket)
        return info

    def counters(self) -> dict:
        keys = ("batches", "graphs", "vertices", "edges", "busy_ns", "queued", "lane_ns", "bytes_in_use",
                "bytes_peak", "lanes")
        out = np.zeros(len(keys), np.int64)
        check(_lib.lib().ispan_server_counters(self._h, out.ctypes.data, len(keys)), "counters")
        return dict(zip(keys, (int(x) for x in out)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().ispan_server_destroy(self._h)
            self._h = None
            self._keep.clear()
            self._done.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def condensation(fw_beg, fw_adj, labels, stream=None) -> np.ndarray:
    """The SCC DAG of a device graph (torch CUDA tensors: forward offsets and
    adjacency) given its device labels: an (n, 2) int64 array of distinct
    (source label, target label) pairs, sorted."""
    V = fw_beg.numel() - 1
    g = _lib.Csr(V, fw_adj.numel(), _ptr(fw_beg), _ptr(fw_beg), _ptr(fw_adj), _ptr(fw_adj),
                 fw_beg.element_size(), 1)
    n = C.c_int64()
    h = C.c_void_p(0 if stream is None else int(getattr(stream, "cuda_stream", stream)))
    check(_lib.lib().ispan_condense(C.byref(g), C.c_void_p(_ptr(labels)), None, 0, C.byref(n), h), "ispan_condense")
    out = np.empty(max(n.value, 1), np.uint64)
    check(_lib.lib().ispan_condense(C.byref(g), C.c_void_p(_ptr(labels)), C.c_void_p(out.ctypes.data), n.value,
                                    C.byref(n), h), "ispan_condense")
    out = out[:n.value]
    return np.stack([(out >> np.uint64(32)).astype(np.int64), (out & np.uint64(0xffffffff)).astype(np.int64)], 1)


def scc(csr: CSR, **kw):
    """One-shot convenience: canonical labels and statistics of a host CSR."""
    with Context(max(csr.V, 1), max(csr.E, 1)) as ctx:
        return ctx.run_csr(csr, **kw)


# ---------------------------------------------------------------------------
# mirror of the reference's interface

@dataclass
class graph:
    """The reference's ``class graph`` (src/graph.h:9-31): public CSR arrays."""

    fw_beg_pos: np.ndarray
    fw_csr: np.ndarray
    bw_beg_pos: np.ndarray
    bw_csr: np.ndarray
    vert_count: int
    edge_count: int


def graph_load(fw_beg_file, fw_csr_file, bw_beg_file, bw_csr_file, avg_time=None) -> graph:
    """src/load_print.cpp:6-22: read the four CSR files and zero avg_time[15].
    Raises (OSError / ValueError) where the reference exits or asserts."""
    c = read_bin(fw_beg_file, fw_csr_file, bw_beg_file, bw_csr_file)
    if avg_time is not None:
        for i in range(15):
            avg_time[i] = 0.0
    return graph(c.fw_beg, c.fw_adj, c.bw_beg, c.bw_adj, c.V, c.E)


_ctx_cache: dict = {}


def _context_for(V, E) -> Context:
    c = _ctx_cache.get("ctx")
    if c is None or c.max_V < V or c.max_E < E:
        if c is not None:
            c.close()
        c = Context(max(V, 1), max(E, 1))
        _ctx_cache["ctx"] = c
    return c


def get_scc_result(scc_id: np.ndarray, vert_count: int) -> dict:
    """src/load_print.cpp:24-60: class report over the reference's codes
    (1 giant, -1/-2/-3/-4 trims, otherwise one group per value), printed in
    the reference's format; returns the counts.  Replace this function (like
    the reference's link-time hook) to consume the codes elsewhere."""
    s = np.asarray(scc_id[:vert_count + 1])
    largest = int((s == 1).sum())
    size_1 = int((s == -1).sum())
    size_2 = int((s == -2).sum())
    size_3 = int((s == -3).sum()) + int((s == -4).sum())
    others = len(np.unique(s[~np.isin(s, [1, -1, -2, -3, -4])]))
    total = 1 + size_1 + size_2 // 2 + size_3 // 3 + others
    print("\nResult:\nlargest, %d\ntrimmed size_1, %d\ntrimmed size_2, %d\ntrimmed size_3, %d\nothers, %d\n"
          "total, %d" % (largest, size_1, size_2 // 2, size_3 // 3, others, total))
    return dict(largest=largest, size_1=size_1, size_2=size_2 // 2, size_3=size_3 // 3, others=others, total=total)


def scc_detection(g: graph, alpha: int, beta: int, gamma: int, theta: float, thread_count: int,
                  avg_time: list, result_hook=None) -> np.ndarray:
    """src/scc_core.cpp:27: detect the SCCs of ``g`` on the GPU.

    ``thread_count`` is accepted for signature parity (the work runs on the
    GPU).  Stage times are accumulated into ``avg_time`` in seconds with the
    reference's slot meanings (0 trim, 1 elephant, 2 mice, 3 total, 4 trim
    size_1, 5 trim size_2, 6 pivot, 7 FW, 8 BW, 9 WCC, 10 mice FW-BW, 13 trim
    size_3).  The reference-convention codes (V+1 entries) go to
    ``result_hook`` (default :func:`get_scc_result`), as at
    src/scc_core.cpp:1076.  Returns the canonical labels."""
    ctx = _context_for(g.vert_count, g.edge_count)
    labels, st = ctx.run(g.fw_beg_pos, g.fw_csr, g.bw_beg_pos, g.bw_csr, V=g.vert_count, alpha=alpha,
                         beta=beta, gamma=gamma, theta=theta, stage_times=True)
    for i in (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 13):  # the reference's slots only
        avg_time[i] += st["stage_ms"][i] / 1000.0
    codes = ctx.ref_codes(g.vert_count)
    (result_hook or get_scc_result)(codes, g.vert_count)
    return labels


def print_time_result(run_times: int, avg_time: list) -> None:
    """src/load_print.cpp:62-92: mean stage times in ms, reference format."""
    if run_times <= 0:
        return
    t = [a / run_times * 1000 for a in avg_time]
    print("\nAverage Time Consumption for Running %d Times (ms)" % run_times)
    for name, i in (("Trim", 0), ("Elephant SCC", 1), ("Mice SCC", 2), ("Total time", 3)):
        print("%s, %.3f" % (name, t[i]))
    print("\n------Details------")
    for name, i in (("Trim size_1", 4), ("Pivot selection", 6), ("FW BFS", 7), ("BW BFS", 8),
                    ("Trim size_2", 5), ("Trim size_3", 13), ("Wcc", 9), ("Mice fw-bw", 10)):
        print("%s, %.3f" % (name, t[i]))

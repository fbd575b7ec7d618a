"""ctypes wrapper over the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline/reference
legs import this module, and only as the checker or the timed CPU baseline.
The product (the ispan_b200 package and its CUDA library) never imports it.

* ``ispan``      serial restatement of iSpan's pipeline (ispan_oracle.c).
* ``tarjan``     exact SCC partition (iterative Tarjan), optionally split by a
                 grouping key, which canonicalises the reference's raw codes.
* ``ref_run``    the reference's own OpenMP ``scc_detection`` compiled from
                 its unmodified sources into _ref/libispan_ref.so (present only
                 where the reference tree was available at build time).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libispan_ref.so")
REF_BIN = os.path.join(HERE, "_ref", "ispan")
REF_DUMP = os.path.join(HERE, "_ref", "ispan_dump")


class _Graph(C.Structure):
    _fields_ = [("V", C.c_int64), ("E", C.c_int64),
                ("fw_beg", C.c_void_p), ("bw_beg", C.c_void_p),
                ("fw_adj", C.c_void_p), ("bw_adj", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "pivot", "fq_after_trim1", "fw_size", "giant_size", "n_trim1", "n_trim2",
        "n_trim3_cycle", "n_trim3_hub", "n_mice_vertices", "n_mice_scc", "n_wcc", "scc_count")] + \
        [("fw_levels", C.c_int32), ("bw_levels", C.c_int32), ("trim1_passes", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_ref = None


def build(ref: bool = False) -> None:
    """Compile liboracle.so (and the reference build when ``ref``)."""
    subprocess.run(["make", "-s", "-C", HERE] + (["ref"] if ref else []), check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oc_ispan.argtypes = [C.POINTER(_Graph), C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                               C.c_void_p, C.c_void_p, C.POINTER(Stats)]
        L.oc_tarjan.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_void_p]
        L.oc_tarjan.restype = C.c_int64
        L.oc_histogram.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64]
        L.oc_histogram.restype = C.c_int64
        L.oc_count.argtypes = [C.c_void_p, C.c_int64]
        L.oc_count.restype = C.c_int64
        _lib = L
    return _lib


def _graph(csr):
    """Keep int64 copies of the offsets alive alongside the struct."""
    fb = np.ascontiguousarray(csr.fw_beg, np.int64)
    bb = np.ascontiguousarray(csr.bw_beg, np.int64)
    fa = np.ascontiguousarray(csr.fw_adj, np.int32)
    ba = np.ascontiguousarray(csr.bw_adj, np.int32)
    g = _Graph(csr.V, csr.E, fb.ctypes.data, bb.ctypes.data, fa.ctypes.data, ba.ctypes.data)
    return g, (fb, bb, fa, ba)


class NonTerminating(RuntimeError):
    """The reproduced reference run would loop forever."""


Q2, Q3, Q4, Q8 = 1, 2, 4, 8
QUIRKS_ALL = Q2 | Q3 | Q4 | Q8


def ispan(csr, alpha=30, beta=200, gamma=10, theta=0.1, quirks=0):
    """Serial iSpan restatement -> (labels[V], codes[V+1], stats dict).
    ``quirks`` re-enables reference quirks (QUIRKS_ALL reproduces the
    reference's serial raw codes)."""
    g, keep = _graph(csr)
    labels = np.empty(max(csr.V, 1), np.int32)
    codes = np.empty(csr.V + 1, np.int32)
    st = Stats()
    rc = lib().oc_ispan(C.byref(g), alpha, beta, gamma, theta, quirks, labels.ctypes.data,
                        codes.ctypes.data, C.byref(st))
    if rc == -2:
        raise NonTerminating("the reference's serial run would not terminate (Q2, pivot 0)")
    if rc:
        raise MemoryError("oc_ispan failed")
    return labels[:csr.V], codes, st.as_dict()


def tarjan(csr, key=None):
    """Exact canonical (min-id) SCC labels; ``key`` splits by group first."""
    g, keep = _graph(csr)
    labels = np.empty(max(csr.V, 1), np.int32)
    k = None if key is None else np.ascontiguousarray(key[:csr.V], np.int32)
    n = lib().oc_tarjan(C.byref(g), None if k is None else k.ctypes.data, labels.ctypes.data)
    if n < 0:
        raise MemoryError("oc_tarjan failed")
    return labels[:csr.V]


def histogram(labels):
    """Sparse SCC size histogram: dict size -> count."""
    labels = np.ascontiguousarray(labels, np.int32)
    V = len(labels)
    cap = 1 << 16
    sizes = np.empty(cap, np.int64)
    counts = np.empty(cap, np.int64)
    n = lib().oc_histogram(labels.ctypes.data, V, sizes.ctypes.data, counts.ctypes.data, cap)
    if n > cap:
        sizes = np.empty(n, np.int64)
        counts = np.empty(n, np.int64)
        n = lib().oc_histogram(labels.ctypes.data, V, sizes.ctypes.data, counts.ctypes.data, n)
    return {int(s): int(c) for s, c in zip(sizes[:n], counts[:n])}


def scc_count(labels):
    labels = np.ascontiguousarray(labels, np.int32)
    return int(lib().oc_count(labels.ctypes.data, len(labels)))


def canon_codes(csr, codes):
    """Canonicalise the reference's raw scc_id codes: group by code (each -1
    vertex alone), split every group into the SCCs of its induced subgraph,
    label each with its minimum vertex id."""
    key = np.asarray(codes[:csr.V], np.int64)
    k = np.where(key == -1, -1, key)
    # remap to int32 keys that keep -1 for singletons
    uniq, inv = np.unique(k, return_inverse=True)
    k32 = inv.astype(np.int32)
    if (uniq == -1).any():
        k32[k == -1] = -1
    return tarjan(csr, k32)


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_LIB)
        L.ispan_ref_run.argtypes = [C.c_int32, C.c_int32] + [C.c_void_p] * 4 + \
            [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_int]
        L.ispan_ref_run.restype = C.c_int
        _ref = L
    return _ref


def ref_run(csr, threads, alpha=30, beta=200, gamma=10, theta=0.1, quiet=True):
    """Run the reference's own scc_detection in-process on int32 CSR arrays.
    Returns (scc_id codes [V+1], avg_time[15] in seconds for this one run)."""
    if csr.E >= 2**31 or csr.V >= 2**31 - 1:
        raise ValueError("the reference's int32 index_t cannot hold this graph")
    fb = np.ascontiguousarray(csr.fw_beg, np.int32)
    bb = np.ascontiguousarray(csr.bw_beg, np.int32)
    fa = np.ascontiguousarray(csr.fw_adj, np.int32)
    ba = np.ascontiguousarray(csr.bw_adj, np.int32)
    out = np.zeros(csr.V + 1, np.int32)
    t = np.zeros(15, np.float64)
    ref_lib().ispan_ref_run(csr.V, csr.E, fb.ctypes.data, fa.ctypes.data, bb.ctypes.data,
                            ba.ctypes.data, threads, alpha, beta, gamma, theta,
                            t.ctypes.data, out.ctypes.data, 1 if quiet else 0)
    return out, t

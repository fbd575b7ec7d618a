"""Seeded synthetic graphs generated on the GPU (ctypes over include/ispan_gen.h).

The shapes follow the benchmark configurations: R-MAT, a social-network
stand-in for Twitter (41.6 M vertices, 1.47 B edges, ~80 % giant SCC), a
web-crawl shape (giant + trivial + planted mid-size SCCs in a DAG), and a
batch of independent graphs as one disjoint union.  The graphs are seeded
synthetic stand-ins; no dataset is reproduced.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .graphs import CSR

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libispan_gen.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ispan_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, I64, I32, D = C.c_void_p, C.c_int64, C.c_int32, C.c_double
        L.ispan_gen_rmat.argtypes = [C.c_int, C.c_int, C.c_int, D, D, D, C.c_uint64, C.c_int, C.POINTER(P)]
        L.ispan_gen_social.argtypes = [C.c_int, I64, I64, D, D, D, I64, I64, I64, I32, C.c_uint64, C.POINTER(P)]
        L.ispan_gen_web.argtypes = [C.c_int, I64, I64, D, D, I32, I32, C.c_uint64, C.POINTER(P)]
        L.ispan_gen_batch.argtypes = [C.c_int, I32, I64, I64, I32, I32, I32, C.c_uint64, P, C.POINTER(P)]
        L.ispan_gen_info.argtypes = [P, C.POINTER(I64), C.POINTER(I64)]
        L.ispan_gen_copy.argtypes = [P, P, P, P, P, I32, I32]
        L.ispan_gen_planted_labels.argtypes = [P, P]
        L.ispan_gen_from_edges.argtypes = [C.c_int, I64, P, P, I64, I32, C.POINTER(P)]
        L.ispan_gen_device_ptrs.argtypes = [P, C.POINTER(P), C.POINTER(P), C.POINTER(P), C.POINTER(P)]
        L.ispan_gen_free.argtypes = [P]
        L.ispan_gen_extract.argtypes = [P, I64, I64, P, P, P, P, I32, C.POINTER(I64)]
        _lib = L
    return _lib


class DeviceGraph:
    """A generated graph resident on the GPU (int64 offsets, int32 ids)."""

    def __init__(self, handle, vbase=None):
        self._h = handle
        V, E = C.c_int64(), C.c_int64()
        lib().ispan_gen_info(handle, C.byref(V), C.byref(E))
        self.V, self.E = V.value, E.value
        self.vbase = vbase
        p = [C.c_void_p() for _ in range(4)]
        lib().ispan_gen_device_ptrs(handle, *[C.byref(x) for x in p])
        self.ptrs = tuple(x.value or 0 for x in p)  # fw_beg, fw_adj, bw_beg, bw_adj

    def to_host(self, offset_dtype=np.int64) -> CSR:
        ob = np.dtype(offset_dtype).itemsize
        fb = np.empty(self.V + 1, offset_dtype)
        bb = np.empty(self.V + 1, offset_dtype)
        fa = np.empty(max(self.E, 1), np.int32)
        ba = np.empty(max(self.E, 1), np.int32)
        rc = lib().ispan_gen_copy(self._h, fb.ctypes.data, fa.ctypes.data, bb.ctypes.data, ba.ctypes.data, ob, 0)
        if rc:
            raise RuntimeError(f"ispan_gen_copy failed ({rc})")
        return CSR(self.V, self.E, fb, fa[:self.E], bb, ba[:self.E])

    def planted_labels(self):
        """The planted SCC partition as canonical labels (CUDA int32 tensor),
        or None for generators without one (R-MAT, batch)."""
        import torch
        out = torch.empty(max(self.V, 1), dtype=torch.int32, device="cuda")
        rc = lib().ispan_gen_planted_labels(self._h, out.data_ptr())
        if rc == -4:
            return None
        if rc:
            raise RuntimeError(f"ispan_gen_planted_labels failed ({rc})")
        return out[:self.V]

    def to_pinned(self):
        """Copies in pinned host memory as CPU tensors (int64 offsets)."""
        import torch
        fb = torch.empty(self.V + 1, dtype=torch.int64, pin_memory=True)
        bb = torch.empty(self.V + 1, dtype=torch.int64, pin_memory=True)
        fa = torch.empty(max(self.E, 1), dtype=torch.int32, pin_memory=True)
        ba = torch.empty(max(self.E, 1), dtype=torch.int32, pin_memory=True)
        rc = lib().ispan_gen_copy(self._h, fb.data_ptr(), fa.data_ptr(), bb.data_ptr(), ba.data_ptr(), 8, 0)
        if rc:
            raise RuntimeError(f"ispan_gen_copy failed ({rc})")
        return fb, fa[:self.E], bb, ba[:self.E]

    def to_torch(self, offset_dtype="int64"):
        """Copies as CUDA tensors (fw_beg, fw_adj, bw_beg, bw_adj)."""
        import torch
        dt = getattr(torch, offset_dtype)
        fb = torch.empty(self.V + 1, dtype=dt, device="cuda")
        bb = torch.empty(self.V + 1, dtype=dt, device="cuda")
        fa = torch.empty(max(self.E, 1), dtype=torch.int32, device="cuda")
        ba = torch.empty(max(self.E, 1), dtype=torch.int32, device="cuda")
        rc = lib().ispan_gen_copy(self._h, fb.data_ptr(), fa.data_ptr(), bb.data_ptr(), ba.data_ptr(),
                                  fb.element_size(), 1)
        if rc:
            raise RuntimeError(f"ispan_gen_copy failed ({rc})")
        return fb, fa[:self.E], bb, ba[:self.E]

    def extract(self, i, offset_dtype="int32"):
        """Graph i of a batch as CUDA tensors with local ids."""
        import torch
        lo, hi = int(self.vbase[i]), int(self.vbase[i + 1])
        E = C.c_int64()
        rc = lib().ispan_gen_extract(self._h, lo, hi, None, None, None, None, 8, C.byref(E))
        if rc:
            raise RuntimeError(f"ispan_gen_extract failed ({rc})")
        dt = getattr(torch, offset_dtype)
        n, e = hi - lo, E.value
        fb = torch.empty(n + 1, dtype=dt, device="cuda")
        bb = torch.empty(n + 1, dtype=dt, device="cuda")
        fa = torch.empty(max(e, 1), dtype=torch.int32, device="cuda")
        ba = torch.empty(max(e, 1), dtype=torch.int32, device="cuda")
        rc = lib().ispan_gen_extract(self._h, lo, hi, fb.data_ptr(), fa.data_ptr(), bb.data_ptr(), ba.data_ptr(),
                                     fb.element_size(), C.byref(E))
        if rc:
            raise RuntimeError(f"ispan_gen_extract failed ({rc})")
        return fb, fa[:e], bb, ba[:e]

    def free(self):
        if self._h:
            lib().ispan_gen_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _mk(rc, h, what, vbase=None):
    if rc:
        raise RuntimeError(f"{what} failed ({rc})")
    return DeviceGraph(h, vbase)


def rmat(scale=16, edge_factor=16, seed=1, a=0.57, b=0.19, c=0.19, permute=False, device=0) -> DeviceGraph:
    h = C.c_void_p()
    return _mk(lib().ispan_gen_rmat(device, scale, edge_factor, a, b, c, seed, int(permute), C.byref(h)), h,
               "ispan_gen_rmat")


# Twitter-shaped stand-in: sizes of paper Table II (TW), synthetic content.
# `edges` counts sampled edges; duplicates among hub pairs are dropped, which
# leaves ~1.47 B distinct edges at full size.
SOCIAL_TW = dict(n=41_652_231, edges=1_735_000_000, giant_frac=0.8038, gamma_out=2.1, gamma_in=1.9,
                 n_pair=80_112, n_tri=12_198, n_tail=5_320, max_tail=1000)


def social(seed=1, scale=1.0, device=0, **kw) -> DeviceGraph:
    """Social-network shape; ``scale`` shrinks every count proportionally."""
    p = dict(SOCIAL_TW)
    p.update(kw)
    if scale != 1.0:
        for k in ("n", "edges", "n_pair", "n_tri", "n_tail"):
            p[k] = max(1, int(p[k] * scale))
    h = C.c_void_p()
    rc = lib().ispan_gen_social(device, p["n"], p["edges"], p["giant_frac"], p["gamma_out"], p["gamma_in"],
                                p["n_pair"], p["n_tri"], p["n_tail"], p["max_tail"], seed, C.byref(h))
    return _mk(rc, h, "ispan_gen_social")


WEB = dict(n=700_000_000, edges=3_300_000_000, giant_frac=0.35, trivial_frac=0.50, min_scc=10, max_scc=10_000)


def web(seed=1, scale=1.0, device=0, **kw) -> DeviceGraph:
    p = dict(WEB)
    p.update(kw)
    if scale != 1.0:
        p["n"], p["edges"] = int(p["n"] * scale), int(p["edges"] * scale)
    h = C.c_void_p()
    rc = lib().ispan_gen_web(device, p["n"], p["edges"], p["giant_frac"], p["trivial_frac"], p["min_scc"],
                             p["max_scc"], seed, C.byref(h))
    return _mk(rc, h, "ispan_gen_web")


def from_edges(V: int, src, dst, device=0) -> DeviceGraph:
    """Both CSR directions of an edge list on the GPU (numpy or CUDA int32
    arrays); sorted, self-loops and duplicates dropped."""
    import numpy as _np
    on_dev = hasattr(src, "is_cuda") and src.is_cuda
    if not on_dev:
        src = _np.ascontiguousarray(src, _np.int32)
        dst = _np.ascontiguousarray(dst, _np.int32)
        ps, pd = src.ctypes.data, dst.ctypes.data
        m = len(src)
    else:
        ps, pd, m = src.data_ptr(), dst.data_ptr(), src.numel()
    h = C.c_void_p()
    rc = lib().ispan_gen_from_edges(device, int(V), ps, pd, int(m), 1 if on_dev else 0, C.byref(h))
    return _mk(rc, h, "ispan_gen_from_edges")


def batch(nseg=4096, vmin=1000, vmax=1_000_000, ef_min=8, ef_max=32, max_cycle=1000, seed=1, device=0):
    vb = np.zeros(nseg + 1, np.int64)
    h = C.c_void_p()
    rc = lib().ispan_gen_batch(device, nseg, vmin, vmax, ef_min, ef_max, max_cycle, seed, vb.ctypes.data,
                               C.byref(h))
    return _mk(rc, h, "ispan_gen_batch", vbase=vb)

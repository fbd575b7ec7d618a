"""ctypes binding of include/ispan_b200.h (libispan_b200.so, built in-tree).

The product path has no CPU fallback: if the CUDA library is missing or no
GPU is visible, loading or running raises instead of computing elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# ISPAN_CHECKED=1 loads the self-checking build (range checks on every index)
LIB_PATH = os.path.join(HERE, "libispan_b200_checked.so" if os.environ.get("ISPAN_CHECKED") == "1"
                        else "libispan_b200.so")

ISPAN_OK = 0
ERRORS = {-1: "ISPAN_ERR_ARG", -2: "ISPAN_ERR_NOMEM", -3: "ISPAN_ERR_CUDA", -4: "ISPAN_ERR_TIMEOUT",
          -5: "ISPAN_ERR_INTERNAL", -6: "ISPAN_ERR_NODEV", -7: "ISPAN_ERR_CAPACITY", -8: "ISPAN_ERR_BUSY"}

F_LABELS_ON_DEVICE = 1
F_NO_GRAPH = 2
F_STAGE_TIMES = 4
F_NO_L2_WINDOW = 8
F_VALIDATE = 16
F_EXACT_STATS = 32
F_REVERSE_ATOMIC = 64
NOALLOC_MAX_V = 65536


class IspanError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        name = ERRORS.get(code, str(code))
        msg = _lib.ispan_strerror(code).decode() if _lib is not None else name
        super().__init__(f"{what}: {name} ({msg})" if what else f"{name} ({msg})")


class Csr(C.Structure):
    _fields_ = [("V", C.c_int64), ("E", C.c_int64), ("fw_beg", C.c_void_p), ("bw_beg", C.c_void_p),
                ("fw_adj", C.c_void_p), ("bw_adj", C.c_void_p), ("offset_bytes", C.c_int32),
                ("on_device", C.c_int32)]


class Params(C.Structure):
    _fields_ = [("alpha", C.c_int32), ("beta", C.c_int32), ("gamma", C.c_int32), ("theta", C.c_double),
                ("flags", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("stage_ms", C.c_double * 16)] + [(n, C.c_int64) for n in (
        "scc_count", "giant_size", "n_trim1", "n_trim2", "n_trim3", "n_mice_vertices", "n_mice_scc", "n_wcc",
        "fw_size", "fw_levels", "bw_levels", "residual", "color_rounds", "local_wcc", "trim_rounds",
        "fw_edges", "bw_edges")] + [
        ("hist_size", C.c_void_p), ("hist_count", C.c_void_p), ("hist_cap", C.c_int64), ("hist_n", C.c_int64),
        ("resid_edges", C.c_int64), ("peeled_residual", C.c_int64), ("peeled_residual_edges", C.c_int64)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("stage_ms", "hist_size", "hist_count")}
        d["stage_ms"] = list(self.stage_ms)
        return d


class Tuning(C.Structure):
    _fields_ = [("async_v", C.c_int64), ("async_e", C.c_int64), ("async_deg", C.c_int32),
                ("bfs_ctas_per_sm", C.c_int32), ("color_levels", C.c_int32), ("color_pivots", C.c_int32),
                ("color_compact", C.c_int32), ("pair_searches", C.c_int32),
                ("tiny_residual", C.c_int32), ("pdl", C.c_int32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_batch_graphs", C.c_int32), ("n_slots", C.c_int32),
                ("reserved", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("max_batch_V", C.c_int64), ("max_batch_E", C.c_int64), ("max_wait_us", C.c_int64),
                ("max_pending", C.c_int64), ("params", Params)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("batch_graphs", C.c_int32), ("batch_id", C.c_int64),
                ("t_submit_ns", C.c_int64), ("t_start_ns", C.c_int64), ("t_done_ns", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    """Load the engine; raise if it was not built (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m ispan_b200.build`")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.ispan_ctx_create.argtypes = [C.c_int, C.c_int64, C.c_int64, C.POINTER(P)]
        L.ispan_ctx_destroy.argtypes = [P]
        L.ispan_ctx_set_stream.argtypes = [P, P]
        L.ispan_ctx_bytes.argtypes = [C.c_int64, C.c_int64]
        L.ispan_ctx_bytes.restype = C.c_int64
        L.ispan_scc_run.argtypes = [P, C.POINTER(Csr), C.POINTER(Params), P, C.POINTER(Stats)]
        L.ispan_scc_run_batch.argtypes = [P, C.POINTER(Csr), C.c_int32, P, C.POINTER(Params), P,
                                          C.POINTER(Stats)]
        L.ispan_ctx_set_tuning.argtypes = [P, C.POINTER(Tuning)]
        L.ispan_ctx_get_tuning.argtypes = [P, C.POINTER(Tuning)]
        L.ispan_scc_run_graphs.argtypes = [P, C.POINTER(Csr), C.c_int32, P, C.POINTER(Params),
                                           C.POINTER(Stats)]
        L.ispan_graphs_pack.argtypes = [P, C.POINTER(Csr), C.c_int32]
        L.ispan_graphs_run.argtypes = [P, C.POINTER(Csr), C.c_int32, P, C.POINTER(Params), C.POINTER(Stats)]
        L.ispan_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(P)]
        L.ispan_server_limits.argtypes = [P, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                          C.POINTER(C.c_int32)]
        L.ispan_server_submit.argtypes = [P, C.POINTER(Csr), P, C.POINTER(C.c_int64)]
        L.ispan_server_poll.argtypes = [P, C.c_int64, C.POINTER(RequestInfo)]
        L.ispan_server_wait.argtypes = [P, C.c_int64, C.c_int64, C.POINTER(RequestInfo)]
        L.ispan_server_counters.argtypes = [P, P, C.c_int32]
        L.ispan_server_destroy.argtypes = [P]
        L.ispan_shard_expand.argtypes = [C.POINTER(Csr), C.c_int64, C.c_int64, P, P, P, P, P]
        L.ispan_shard_expand_queue.argtypes = [C.POINTER(Csr), C.c_int64, C.c_int64, P, P, P, P, P, P]
        L.ispan_shard_collect.argtypes = [C.c_int64, C.c_int64, P, P, P, P, P]
        L.ispan_condense.argtypes = [C.POINTER(Csr), P, P, C.c_int64, C.POINTER(C.c_int64), P]
        L.ispan_ref_codes.argtypes = [P, P]
        L.ispan_debug_trace.argtypes = [P, P, C.c_int64]
        L.ispan_debug_barrier_timeout.argtypes = [P, C.c_int64]
        L.ispan_scc_small_noalloc.argtypes = [C.POINTER(Csr), P, P]
        L.ispan_strerror.argtypes = [C.c_int]
        L.ispan_strerror.restype = C.c_char_p
        L.ispan_version.restype = C.c_char_p
        _lib = L
    return _lib


SYMBOLS = ("ispan_ctx_create", "ispan_ctx_destroy", "ispan_ctx_set_stream", "ispan_ctx_bytes", "ispan_scc_run",
           "ispan_scc_run_batch", "ispan_scc_run_graphs", "ispan_graphs_pack", "ispan_graphs_run", "ispan_ctx_set_tuning", "ispan_ctx_get_tuning", "ispan_server_create", "ispan_server_limits",
           "ispan_server_submit", "ispan_server_poll", "ispan_server_wait", "ispan_server_counters",
           "ispan_server_destroy", "ispan_condense", "ispan_shard_expand", "ispan_shard_expand_queue", "ispan_shard_collect", "ispan_ref_codes", "ispan_debug_trace", "ispan_debug_barrier_timeout", "ispan_scc_small_noalloc",
           "ispan_strerror", "ispan_version")


def check(rc: int, what: str = "") -> None:
    if rc != ISPAN_OK:
        raise IspanError(rc, what)

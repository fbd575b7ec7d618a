"""The reference's own OpenMP pipeline built with 64-bit integer types --
TEST INFRASTRUCTURE (the CPU baseline of graphs with 2^31 edges or more).

``oracle/Makefile ref64`` compiles the unmodified reference sources with the
authors' own wide typedefs (src/util.h:12-21: index_t, vertex_t, depth_t and
color_t as long) and its DEBUG progress prints on (src/util.h:27) into
_ref/libispan_ref64.so; ``run`` calls its scc_detection in-process.

As a script it is the wide reference run that bench.py times on a graph held
in four raw files (int64 offsets, int32 ids): it widens the arrays to the
build's 64-bit types, prints ``PIPELINE START`` and runs the pipeline, whose
DEBUG lines report each stage as it finishes (src/scc_core.cpp:254-914) and
whose OUTPUT_TIME lines (src/scc_core.cpp:1062-1068) close a finished run.
The caller enforces the wall-clock cap (the reference's small-SCC stage is
superlinear on DAGs of planted SCCs and may not finish).

    python oracle/ref_wide.py <V> <E> <fw_beg> <fw_adj> <bw_beg> <bw_adj> <threads>
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libispan_ref64.so")
PARAMS = (30, 200, 10, 0.1)  # src/bash_one.sh:4
# host bytes the wide run holds per vertex and per edge: the CSR in 64-bit
# types (2 offsets, 2 ids per edge) plus scc_detection's own arrays (8 per-vertex
# arrays of 8 bytes, src/scc_core.cpp:56-93, and its per-thread queues of
# 5 V / T entries each, :166)
BYTES_PER_VERTEX = 2 * 8 + 8 * 8 + 5 * 8
BYTES_PER_EDGE = 2 * 8


def host_bytes(V: int, E: int) -> int:
    return BYTES_PER_VERTEX * V + BYTES_PER_EDGE * E


def _lib():
    L = C.CDLL(LIB)
    P = C.c_void_p
    L.ispan_ref_run64.argtypes = [C.c_int64, C.c_int64, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_double, P, P, C.c_int]
    L.ispan_ref_run64.restype = C.c_int
    return L


def run(fw_beg, fw_adj, bw_beg, bw_adj, threads, quiet=True):
    """The wide reference on host arrays -> (scc_id codes [V+1] int64,
    avg_time[15] in seconds)."""
    V, E = len(fw_beg) - 1, len(fw_adj)
    a = [np.ascontiguousarray(x, np.int64) for x in (fw_beg, fw_adj, bw_beg, bw_adj)]
    codes = np.zeros(V + 1, np.int64)
    t = np.zeros(15, np.float64)
    _lib().ispan_ref_run64(V, E, a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, a[3].ctypes.data,
                           threads, *PARAMS, t.ctypes.data, codes.ctypes.data, 1 if quiet else 0)
    return codes, t


def main(argv):
    V, E = int(argv[0]), int(argv[1])
    paths, threads = argv[2:6], int(argv[6])
    t0 = time.time()
    arrs = []
    for p, dt, n in zip(paths, (np.int64, np.int32, np.int64, np.int32), (V + 1, E, V + 1, E)):
        src = np.memmap(p, dtype=dt, mode="r", shape=(n,))
        arrs.append(np.array(src, dtype=np.int64))  # the build's 64-bit types
        del src
        os.unlink(p)  # the file's memory is freed once widened
    print(f"LOADED {time.time() - t0:.1f} s", flush=True)
    L = _lib()
    # the pipeline's own printf lines reach the log as they are printed (a
    # killed run keeps the stages it finished): line-buffered C stdout
    libc = C.CDLL(None)
    libc.setvbuf(C.c_void_p.in_dll(libc, "stdout"), None, 1, 0)  # _IOLBF
    t = np.zeros(15, np.float64)
    print("PIPELINE START", flush=True)
    t1 = time.time()
    L.ispan_ref_run64(V, E, *[x.ctypes.data for x in arrs], threads, *PARAMS, t.ctypes.data, None, 0)
    print(f"PIPELINE DONE {time.time() - t1:.3f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])

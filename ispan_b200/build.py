"""Build the CUDA libraries of the package in-tree (sm_100a only).

    python -m ispan_b200.build        # or ispan_b200.build.build()

Produces ``ispan_b200/libispan_b200.so`` (the SCC engine behind
include/ispan_b200.h) and ``ispan_b200/libispan_gen.so`` (device graph
generators behind include/ispan_gen.h).  nvcc cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC,-O3",
         "-shared", "-I" + os.path.join(ROOT, "include")]

TARGETS = {
    "libispan_b200.so": (["pipeline.cu", "noalloc.cu", "server.cu", "condense.cu", "shard.cu"], ["common.cuh", "bfs.cuh", "stages.cuh", "pack.cuh", "compact.cuh", "tiny.cuh", "transpose.cuh", "lane.h"], []),
    "libispan_gen.so": (["gen.cu"], [], []),
}
# self-checking variant: range checks on every index, first violation reported
CHECKED = {"libispan_b200_checked.so": (["pipeline.cu", "noalloc.cu", "server.cu", "condense.cu", "shard.cu"], ["common.cuh", "bfs.cuh", "stages.cuh", "pack.cuh", "compact.cuh", "tiny.cuh", "transpose.cuh", "lane.h"],
                                        ["-DISPAN_CHECKED"])}


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = srcs + [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))]
    return any(os.path.getmtime(s) > t for s in deps if os.path.exists(s))


def build(force: bool = False, verbose: bool = False, extra=(), checked: bool = False) -> list[str]:
    outs = []
    targets = dict(TARGETS)
    if checked:
        targets.update(CHECKED)
    for lib, (srcs, hdrs, defs) in targets.items():
        src = [os.path.join(CSRC, s) for s in srcs]
        if not all(os.path.exists(s) for s in src):
            continue
        out = os.path.join(HERE, lib)
        if force or _stale(out, src + [os.path.join(CSRC, h) for h in hdrs]):
            cmd = [NVCC, *ARCH, *FLAGS, *defs, *extra, *src, "-o", out]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        outs.append(out)
    return outs


if __name__ == "__main__":
    print("\n".join(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv,
                          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else [])))

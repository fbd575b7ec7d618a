"""Regenerate the golden fixtures in this directory from the reference itself.

Run where the reference tree is present (it is read at build time only):

    make -C oracle ref && python tests/golden/make_golden.py [--rmat16]

For every fixture graph this writes ``<name>.npz`` holding the CSR, the raw
per-vertex ``scc_id`` codes that the reference's unmodified CLI
(src/scc_main.cpp + src/scc_core.cpp, linked with the dump hook
oracle/ref_hook_dump.cpp) hands to get_scc_result, for 1 and 4 OpenMP
threads, the reference's printed class report, and the exact canonical
labels from the independent Tarjan oracle.  ``ref_exact_t1`` /
``ref_exact_t4`` record whether the reference's answer, after splitting its
codes into induced SCCs, equals the exact partition (it does not on some
planted-cycle graphs: stale forward marks in init_fw_sa, src/fw_bw.h:1560).

The plain-pipeline small workload (R-MAT scale 16, edge factor 16,
(a,b,c) = (.57,.19,.19), self-loops and duplicates removed, seeds 1-10) gets
its fixtures in ``rmat16/s<seed>.npz``: the graph is regenerated from its seed
by ispan_b200.graphs.rmat (the fixture keeps a SHA-256 of its arrays to prove
it is the same graph) and only the reference's raw codes (1 and 16 OpenMP
threads) and its printed class report are stored.
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from ispan_b200 import graphs as G  # noqa: E402

PARAMS = ("30", "200", "10", "0.1")  # src/bash_one.sh:4


def fixtures():
    yield "toy", G.toy()
    yield "rmat10_s1", G.rmat(10, 16, 1)
    yield "rmat10_s2_perm", G.rmat(10, 16, 2, permute=True)
    yield "rmat11_ef8_s3", G.rmat(11, 8, 3)
    yield "planted600_s0", G.planted(600, 0, giant_frac=0.3, permute=False)
    yield "planted600_s2", G.planted(600, 2, giant_frac=0.3, permute=True)
    yield "planted1500_s5", G.planted(1500, 5, giant_frac=0.0, permute=True)
    yield "random800", G.random_graph(800, 2400, 7)
    # hand-built corner cases: self-loops, duplicates, 2-cycles (sink and
    # source), both trim-3 shapes, a long cycle, isolated vertices
    e = [(0, 0), (0, 1), (1, 0), (1, 0), (2, 3), (3, 4), (4, 2), (5, 6), (5, 7), (6, 5), (7, 5),
         (8, 9), (9, 10), (10, 11), (11, 12), (12, 8), (12, 2), (1, 5), (13, 13), (14, 1)]
    yield "corners", G.from_edges(16, np.array(e))


CONFIG1_SEEDS = range(1, 11)


def csr_digest(csr):
    import hashlib
    h = hashlib.sha256()
    for a in (csr.fw_beg, csr.fw_adj, csr.bw_beg, csr.bw_adj):
        h.update(np.ascontiguousarray(a, np.int32).tobytes())
    return h.hexdigest()


def config1(tmp):
    os.makedirs(os.path.join(HERE, "rmat16"), exist_ok=True)
    for seed in CONFIG1_SEEDS:
        csr = G.rmat(16, 16, seed)
        exact = oracle.tarjan(csr)
        out = dict(V=csr.V, E=csr.E, seed=seed, sha256=csr_digest(csr))
        for t in (1, 16):
            codes, report = run_cli(csr, os.path.join(tmp, f"rmat16_{seed}"), t)
            out[f"ref_codes_t{t}"] = codes
            out[f"ref_exact_t{t}"] = bool((oracle.canon_codes(csr, codes) == exact).all())
            out[f"ref_report_t{t}"] = report
        np.savez_compressed(os.path.join(HERE, "rmat16", f"s{seed}.npz"), **out)
        print("rmat16", seed, csr.V, csr.E, "ref exact t1/t16:", out["ref_exact_t1"], out["ref_exact_t16"])


def run_cli(csr, d, threads):
    paths = G.write_bin(csr, d)
    dump = os.path.join(d, "sid.bin")
    env = dict(os.environ, ISPAN_DUMP=dump)
    r = subprocess.run([oracle.REF_DUMP, *paths, str(threads), *PARAMS, "1"], env=env,
                       capture_output=True, text=True, timeout=30, check=True)
    r2 = subprocess.run([oracle.REF_BIN, *paths, str(threads), *PARAMS, "1"],
                        capture_output=True, text=True, timeout=30, check=True)
    report = r2.stdout[r2.stdout.index("Result:"):r2.stdout.index("Average")].strip()
    return np.fromfile(dump, np.int32), report


def main():
    if not os.path.exists(oracle.REF_DUMP):
        sys.exit("build the reference first: make -C oracle ref")
    with tempfile.TemporaryDirectory() as tmp:
        if "--rmat16" in sys.argv:
            config1(tmp)
            return
        for name, csr in fixtures():
            exact = oracle.tarjan(csr)
            out = dict(V=csr.V, E=csr.E, fw_beg=csr.fw_beg, fw_adj=csr.fw_adj,
                       bw_beg=csr.bw_beg, bw_adj=csr.bw_adj, exact=exact)
            try:
                oracle.ispan(csr, quirks=oracle.QUIRKS_ALL)
                out["ref_nonterminating"] = False
            except oracle.NonTerminating:
                # vertex 0 pivots a multi-vertex mice SCC; the reference loops
                # forever there (confirmed by running it under a timeout once)
                out["ref_nonterminating"] = True
                np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
                print(name, csr.V, csr.E, "reference does not terminate")
                continue
            for t in (1, 4):
                codes, report = run_cli(csr, os.path.join(tmp, name), t)
                out[f"ref_codes_t{t}"] = codes
                out[f"ref_exact_t{t}"] = bool((oracle.canon_codes(csr, codes) == exact).all())
                out[f"ref_report_t{t}"] = report
            np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
            print(name, csr.V, csr.E, "ref exact t1/t4:", out["ref_exact_t1"], out["ref_exact_t4"])


if __name__ == "__main__":
    main()

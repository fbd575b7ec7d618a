"""Host-side CSR graphs in iSpan's binary format, plus small seeded generators.

The reference stores a directed graph as four raw little-endian files
(src/graph.cpp:2-92): ``fw_begin.bin`` int32[V+1] out-edge offsets,
``fw_adjacent.bin`` int32[E] out-neighbour ids, and ``bw_begin.bin`` /
``bw_adjacent.bin``, the same for in-edges.  The offline converter
(graph_converter/txt_to_bin_fw_int.cpp) writes the forward pair from a text
edge list.  :class:`CSR` holds both directions; offsets may be int32 (the
reference's width) or int64 (for graphs beyond 2^31 edges).

The numpy generators here build the small graphs the CPU tests use; the
full-size benchmark graphs come from the device generators of the CUDA
library (``ispan_b200.gen``).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class CSR:
    """Forward + backward CSR of one directed graph (src/graph.h:9-31)."""

    V: int
    E: int
    fw_beg: np.ndarray  # [V+1] int32 or int64
    fw_adj: np.ndarray  # [E] int32
    bw_beg: np.ndarray
    bw_adj: np.ndarray

    @property
    def offset_bytes(self) -> int:
        return self.fw_beg.dtype.itemsize

    def with_offsets(self, dtype) -> "CSR":
        """Same graph with offsets cast to ``dtype`` (int32 needs E < 2^31)."""
        dt = np.dtype(dtype)
        if dt == np.int32 and self.E >= 2**31:
            raise ValueError("int32 offsets cannot address %d edges" % self.E)
        return CSR(self.V, self.E, self.fw_beg.astype(dt), self.fw_adj,
                   self.bw_beg.astype(dt), self.bw_adj)

    def edges(self) -> np.ndarray:
        """[E, 2] int64 (src, dst) pairs in forward-CSR order."""
        src = np.repeat(np.arange(self.V, dtype=np.int64), np.diff(self.fw_beg.astype(np.int64)))
        return np.stack([src, self.fw_adj.astype(np.int64)], 1)


def from_edges(V: int, edges: np.ndarray, offset_dtype=np.int32, sort: bool = True) -> CSR:
    """Build fw and bw CSR from an [E, 2] edge array (duplicates and self-loops
    are kept as given, like the reference converter)."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    if len(e) and (e.min() < 0 or e.max() >= V):
        raise ValueError("edge endpoint out of range")
    out = []
    for s, t in ((e[:, 0], e[:, 1]), (e[:, 1], e[:, 0])):
        order = np.lexsort((t, s)) if sort else np.argsort(s, kind="stable")
        beg = np.zeros(V + 1, np.int64)
        np.add.at(beg, s + 1, 1)
        beg = np.cumsum(beg)
        out.append((beg.astype(offset_dtype), t[order].astype(np.int32)))
    return CSR(V, len(e), out[0][0], out[0][1], out[1][0], out[1][1])


def dedupe_edges(edges: np.ndarray) -> np.ndarray:
    """Drop self-loops and duplicate edges."""
    e = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    e = e[e[:, 0] != e[:, 1]]
    return np.unique(e, axis=0) if len(e) else e


# --------------------------------------------------------------------------
# reference binary format (src/graph.cpp:10-13 reads int32 offsets and ids)

FILES = ("fw_begin.bin", "fw_adjacent.bin", "bw_begin.bin", "bw_adjacent.bin")


def write_bin(csr: CSR, directory: str, offset_dtype=np.int32) -> list[str]:
    """Write the four reference files; returns their paths in CLI order."""
    os.makedirs(directory, exist_ok=True)
    g = csr.with_offsets(offset_dtype)
    paths = [os.path.join(directory, f) for f in FILES]
    for p, a in zip(paths, (g.fw_beg, g.fw_adj, g.bw_beg, g.bw_adj)):
        a.tofile(p)
    return paths


def read_bin(fw_beg_file: str, fw_csr_file: str, bw_beg_file: str, bw_csr_file: str,
             offset_dtype=np.int32) -> CSR:
    """Load the four files like ``graph::graph`` (src/graph.cpp:2-92):
    V = size(fw_begin)/width - 1, E = size(fw_adjacent)/4.  Raises on a
    missing file, a short file or offsets that do not match the edge arrays,
    where the reference exits or asserts."""
    dt = np.dtype(offset_dtype)
    fw_beg = np.fromfile(fw_beg_file, dt)
    fw_adj = np.fromfile(fw_csr_file, np.int32)
    bw_beg = np.fromfile(bw_beg_file, dt)
    bw_adj = np.fromfile(bw_csr_file, np.int32)
    V, E = len(fw_beg) - 1, len(fw_adj)
    if V < 0 or len(bw_beg) != V + 1 or len(bw_adj) != E:
        raise ValueError("inconsistent CSR file sizes")
    for beg in (fw_beg, bw_beg):
        if beg[0] != 0 or beg[-1] != E or np.any(np.diff(beg.astype(np.int64)) < 0):
            raise ValueError("CSR offsets are not a monotone 0..E sequence")
    return CSR(V, E, fw_beg, fw_adj, bw_beg, bw_adj)


def validate(csr: CSR) -> None:
    """Raise ValueError unless both CSRs are well formed and are transposes."""
    for beg, adj in ((csr.fw_beg, csr.fw_adj), (csr.bw_beg, csr.bw_adj)):
        b = beg.astype(np.int64)
        if len(b) != csr.V + 1 or b[0] != 0 or b[-1] != csr.E or np.any(np.diff(b) < 0):
            raise ValueError("bad offsets")
        if len(adj) != csr.E or (csr.E and (adj.min() < 0 or adj.max() >= csr.V)):
            raise ValueError("bad adjacency")
    if csr.E:
        f = csr.edges()
        fk = np.sort(f[:, 0] * csr.V + f[:, 1])
        src = np.repeat(np.arange(csr.V, dtype=np.int64), np.diff(csr.bw_beg.astype(np.int64)))
        bk = np.sort(csr.bw_adj.astype(np.int64) * csr.V + src)
        if not np.array_equal(fk, bk):
            raise ValueError("bw CSR is not the transpose of fw CSR")


# --------------------------------------------------------------------------
# small seeded generators (CPU tests; the device generators cover full sizes)

def rmat_edges(scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19,
               permute: bool = False) -> np.ndarray:
    """Graph500-style R-MAT: per-bit quadrant sampling, no noise; self-loops
    and duplicates removed.  ``permute`` relabels vertices randomly."""
    rng = np.random.default_rng(seed)
    n, m = 1 << scale, edge_factor << scale
    src = np.zeros(m, np.int64)
    dst = np.zeros(m, np.int64)
    for bit in range(scale):
        r = rng.random(m)
        sb = r >= a + b
        db = ((r >= a) & (r < a + b)) | (r >= a + b + c)
        src |= sb.astype(np.int64) << bit
        dst |= db.astype(np.int64) << bit
    e = np.stack([src, dst], 1)
    if permute:
        p = rng.permutation(n)
        e = p[e]
    return dedupe_edges(e)


def rmat(scale: int, edge_factor: int = 16, seed: int = 1, offset_dtype=np.int32, **kw) -> CSR:
    return from_edges(1 << scale, rmat_edges(scale, edge_factor, seed, **kw), offset_dtype)


def planted_edges(n: int, seed: int, giant_frac: float = 0.3, dag_ef: float = 2.0,
                  max_cycle: int = 60, chords: float = 1.0, permute: bool = True) -> np.ndarray:
    """Random DAG of planted SCCs: an optional giant cycle with random chords,
    then cycles of length 1..max_cycle (with chords), joined by DAG edges that
    go from earlier to later components in a random topological order."""
    rng = np.random.default_rng(seed)
    ids = rng.permutation(n) if permute else np.arange(n)
    comp = np.empty(n, np.int64)
    parts, pos, c = [], 0, 0
    g = int(n * giant_frac)
    if g > 1:
        vs = ids[:g]
        parts.append(np.stack([vs, np.roll(vs, -1)], 1))
        k = g * 3
        parts.append(np.stack([vs[rng.integers(0, g, k)], vs[rng.integers(0, g, k)]], 1))
        comp[vs] = c
        c, pos = c + 1, g
    while pos < n:
        L = int(min(n - pos, rng.choice([1, 1, 1, 2, 2, 3, 3, int(rng.integers(4, max_cycle + 1))])))
        vs = ids[pos:pos + L]
        if L > 1:
            parts.append(np.stack([vs, np.roll(vs, -1)], 1))
            if L > 3 and chords > 0:
                k = int(L * chords)
                parts.append(np.stack([vs[rng.integers(0, L, k)], vs[rng.integers(0, L, k)]], 1))
        comp[vs] = c
        c, pos = c + 1, pos + L
    k = int(n * dag_ef)
    s, t = rng.integers(0, n, k), rng.integers(0, n, k)
    ok = comp[s] < comp[t]
    parts.append(np.stack([s[ok], t[ok]], 1))
    return dedupe_edges(np.concatenate(parts) if parts else np.zeros((0, 2), np.int64))


def planted(n: int, seed: int = 1, offset_dtype=np.int32, **kw) -> CSR:
    return from_edges(n, planted_edges(n, seed, **kw), offset_dtype)


def toy() -> CSR:
    """The reference's toy graph (graph_converter/toy_edge_list.txt): 7
    vertices, 16 edges, SCCs {0,1,2,3,4} and {5,6}."""
    e = np.array([[0, 1], [0, 2], [1, 0], [1, 2], [1, 3], [1, 4], [2, 0], [2, 1], [2, 3],
                  [3, 1], [3, 2], [3, 4], [4, 1], [4, 3], [5, 6], [6, 5]], np.int64)
    return from_edges(7, e)


def random_graph(n: int, m: int, seed: int, self_loops: bool = True, dups: bool = True) -> CSR:
    """Uniform random multigraph (keeps self-loops/duplicates unless told not to)."""
    rng = np.random.default_rng(seed)
    e = rng.integers(0, max(n, 1), (m, 2)) if n else np.zeros((0, 2), np.int64)
    if not self_loops:
        e = e[e[:, 0] != e[:, 1]]
    if not dups:
        e = np.unique(e, axis=0)
    return from_edges(n, e)


def disjoint_union(graphs: list[CSR]) -> tuple[CSR, np.ndarray]:
    """Pack graphs into one CSR with global ids; returns (union, vbase[n+1])."""
    vb = np.zeros(len(graphs) + 1, np.int64)
    for i, g in enumerate(graphs):
        vb[i + 1] = vb[i] + g.V
    parts = [g.edges() + vb[i] for i, g in enumerate(graphs)]
    e = np.concatenate(parts) if parts else np.zeros((0, 2), np.int64)
    off = np.int64 if len(e) >= 2**31 else np.int32
    return from_edges(int(vb[-1]), e, off), vb

/*
 * ispan_gen.h -- seeded synthetic graph generators on the GPU, writing
 * iSpan's CSR layout (fw/bw offsets + int32 adjacency, src/graph.h:9-31).
 *
 * These build the benchmark and test inputs at full size on the device
 * (a 1.5-billion-edge graph does not fit a reasonable host build time).  They
 * have no counterpart in the reference's pipeline; the reference's own
 * converter (graph_converter/txt_to_bin_{fw,bw}_int.cpp) turns a text edge
 * list into the same files.  Every generator sorts, drops self-loops and
 * duplicate edges, and returns a handle that owns the device CSR.
 */
#ifndef ISPAN_GEN_H
#define ISPAN_GEN_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct ispan_gen_graph ispan_gen_graph;

/* Directed R-MAT, Graph500 style: 2^scale vertices, edge_factor * 2^scale
 * sampled edges, per-bit quadrant probabilities (a, b, c, 1-a-b-c), no noise.
 * permute != 0 relabels vertices with a seeded bijection. */
int ispan_gen_rmat(int device, int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                   int permute, ispan_gen_graph **out);

/* Social-network shape: n vertices, about `edges` edges; a giant SCC of
 * giant_frac * n vertices (Chung-Lu core with out/in power-law exponents
 * gamma_out / gamma_in plus a Hamiltonian cycle that makes it strongly
 * connected), size-1 sources/sinks and upstream/downstream vertices,
 * n_pair 2-cycles, n_tri 3-cycles (both shapes), n_tail longer cycles of
 * power-law lengths 4..max_tail; every small cycle is attached to the core
 * in one direction only.  Vertex 0 is always a core vertex. */
int ispan_gen_social(int device, int64_t n, int64_t edges, double giant_frac, double gamma_out,
                     double gamma_in, int64_t n_pair, int64_t n_tri, int64_t n_tail, int32_t max_tail,
                     uint64_t seed, ispan_gen_graph **out);

/* Web-crawl shape: n vertices, about `edges` edges; giant SCC of giant_frac*n
 * (random core + Hamiltonian cycle), trivial_frac*n size-1 sources/sinks, and
 * the rest in planted SCCs of power-law sizes min_scc..max_scc (a cycle plus
 * chords) joined by DAG edges that go from earlier to later SCCs of a random
 * topological order.  Vertex 0 is always a core vertex. */
int ispan_gen_web(int device, int64_t n, int64_t edges, double giant_frac, double trivial_frac,
                  int32_t min_scc, int32_t max_scc, uint64_t seed, ispan_gen_graph **out);

/* Batch of independent graphs as one disjoint union (segmented CSR with
 * global ids): graph i has V_i vertices (log-uniform in [vmin, vmax]); even
 * i are R-MAT-like (edge factor uniform in [ef_min, ef_max]), odd i are
 * random DAGs of planted cycles of lengths 2..max_cycle.  vbase (nseg+1
 * entries) is written to the caller's host array. */
int ispan_gen_batch(int device, int32_t nseg, int64_t vmin, int64_t vmax, int32_t ef_min, int32_t ef_max,
                    int32_t max_cycle, uint64_t seed, int64_t *vbase_out, ispan_gen_graph **out);

/* CSR construction from an edge list (src[i] -> dst[i], i < m, ids in
 * [0, V); host arrays, or device arrays when on_device != 0): both CSR
 * directions, adjacency sorted, self-loops and duplicate edges dropped
 * (neither changes the SCC partition).  The result is a handle like a
 * generator's (copy, device pointers, free).  An id outside [0, V) returns -1.
 * Replaces the reference's offline converter (graph_converter/
 * txt_to_bin_fw_int.cpp, txt_to_bin_bw_int.cpp), which writes the same two
 * CSR directions from a text edge list on the CPU. */
int ispan_gen_from_edges(int device, int64_t V, const int32_t *src, const int32_t *dst, int64_t m,
                         int32_t on_device, ispan_gen_graph **out);

/* sizes of a generated graph */
int ispan_gen_info(const ispan_gen_graph *g, int64_t *V, int64_t *E);

/* Copy the CSR into caller buffers (device memory when to_device != 0, else
 * host), offsets as offset_bytes = 4 or 8 (4 needs E < 2^31); any pointer may
 * be NULL to skip that array. */
int ispan_gen_copy(const ispan_gen_graph *g, void *fw_beg, int32_t *fw_adj, void *bw_beg, int32_t *bw_adj,
                   int32_t offset_bytes, int32_t to_device);

/* Device pointers owned by the handle (int64 offsets), valid until free. */
int ispan_gen_device_ptrs(const ispan_gen_graph *g, const int64_t **fw_beg, const int32_t **fw_adj,
                          const int64_t **bw_beg, const int32_t **bw_adj);

/* One graph of a batch, [vlo, vhi) of a disjoint union, with local ids
 * (minus vlo) into caller device buffers; *E_out gets its edge count (query
 * first with all array pointers NULL). */
int ispan_gen_extract(const ispan_gen_graph *g, int64_t vlo, int64_t vhi, void *fw_beg, int32_t *fw_adj,
                      void *bw_beg, int32_t *bw_adj, int32_t offset_bytes, int64_t *E_out);

/* The SCC partition the social and web generators plant, as canonical
 * labels (minimum vertex id of each planted SCC) into labels[V] (device
 * memory).  By construction it is the graph's exact SCC partition: the
 * core is strongly connected through its Hamiltonian cycle, every small
 * cycle / planted SCC is attached to the rest in one direction only, and
 * sources, sinks and DAG vertices have no path back.  This gives an exact
 * check at full size, where a CPU Tarjan would take minutes.  -4 for
 * generators without a planted partition (R-MAT, batch). */
int ispan_gen_planted_labels(const ispan_gen_graph *g, int32_t *labels);

int ispan_gen_free(ispan_gen_graph *g);

#ifdef __cplusplus
}
#endif
#endif

/*
 * ispan_oracle.h -- CPU oracle for the iSpan SCC pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path (the ispan_b200
 * package, its CUDA library, the drop-in shim) may link, load or call this.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs use it, and only as the checker.
 *
 * Two independent oracles live here:
 *   oc_ispan()   a serial restatement of iSpan's shared-memory pipeline
 *                (src/scc_core.cpp:27-1094 and the stage headers it calls),
 *                one function per reference stage, each citing the reference
 *                file:line it follows.  Reference quirks Q2/Q3/Q4/Q8 (label
 *                collisions, stale fw_sa, int32 degree product, pivot 0 on an
 *                empty residual) are fixed here; each fix is marked "FIX".
 *   oc_tarjan()  an iterative Tarjan SCC, independent of iSpan, used to pin
 *                the restatement and every GPU result to the exact partition.
 *
 * Both emit canonical labels: every vertex gets the minimum vertex id of its
 * strongly connected component.
 */
#ifndef ISPAN_ORACLE_H
#define ISPAN_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* CSR in the reference's layout (src/graph.h:9-31), offsets widened to int64
 * so graphs above 2^31 edges fit. fw = out-edges, bw = in-edges. */
typedef struct {
    int64_t V, E;
    const int64_t *fw_beg, *bw_beg; /* [V+1] */
    const int32_t *fw_adj, *bw_adj; /* [E]   */
} oc_graph;

typedef struct {
    int64_t pivot;          /* elephant pivot (-1 when the worklist was empty) */
    int64_t fq_after_trim1; /* |Q| after trim_1_first + generate_frontier_queue */
    int64_t fw_size;        /* |F|, forward reach of the pivot */
    int64_t giant_size;     /* |S| = |F ∩ B| */
    int64_t n_trim1;        /* vertices labelled by any trim-1 pass */
    int64_t n_trim2;        /* vertices labelled by trim-2 (pairs * 2) */
    int64_t n_trim3_cycle;  /* trim_3_1: A->B->C->A shapes (vertices) */
    int64_t n_trim3_hub;    /* trim_3_2: A<->B, A<->C shapes (vertices) */
    int64_t n_mice_vertices;
    int64_t n_mice_scc;
    int64_t n_wcc;          /* distinct WCC colours entering mice_fw_bw */
    int64_t scc_count;
    int32_t fw_levels, bw_levels;
    int32_t trim1_passes;
} oc_stats;

/* Reference quirks that oc_ispan can reproduce on request, so that with
 * thread_count = 1 its raw codes can be compared with the reference's own
 * serial run bit for bit.  Default (0) fixes all of them. */
#define OC_Q2 1 /* mice label = pivot id (collides with 0 "active", 1 "giant") */
#define OC_Q3 2 /* init_fw_sa resets queue positions, not queue vertices */
#define OC_Q4 4 /* pivot key is a wrapping int32 degree product */
#define OC_Q8 8 /* pivot defaults to vertex 0; BW marks it giant regardless */
#define OC_QUIRKS_ALL (OC_Q2 | OC_Q3 | OC_Q4 | OC_Q8)

/* Serial restatement of scc_detection (src/scc_core.cpp:27-1094).
 * labels: [V] canonical min-id labels.  codes: optional [V+1] array in the
 * reference's scc_id convention (1 giant, -1 size-1, -2 size-2, -3/-4 size-3,
 * otherwise the mice pivot id + 2 so it never collides with a class code;
 * codes[V] = 0 is the reference's phantom slot).  Returns 0, -1 (alloc), or
 * -2 when quirk Q2 is reproduced and vertex 0 becomes the pivot of a mice SCC
 * of two or more vertices: the reference's backward search never terminates
 * there, because a member's new label 0 still reads as unlabelled. */
int oc_ispan(const oc_graph *g, int alpha, int beta, int gamma, double theta, int quirks,
             int32_t *labels, int32_t *codes, oc_stats *st);

/* Exact SCC labels by iterative Tarjan.  If key != NULL, only edges (u,v) with
 * key[u] == key[v] are followed, and vertices whose key is -1 are singletons:
 * this splits a grouping (e.g. the reference's raw scc_id codes) into the SCCs
 * of each group's induced subgraph.  Returns the number of components or -1. */
int64_t oc_tarjan(const oc_graph *g, const int32_t *key, int32_t *labels);

/* Sparse size histogram of canonical labels: writes up to cap (size, count)
 * pairs sorted by size; returns the number of distinct sizes. */
int64_t oc_histogram(const int32_t *labels, int64_t V, int64_t *sizes,
                     int64_t *counts, int64_t cap);

/* Number of distinct canonical components (vertices with labels[v] == v). */
int64_t oc_count(const int32_t *labels, int64_t V);

#ifdef __cplusplus
}
#endif
#endif

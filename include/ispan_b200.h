/*
 * ispan_b200.h -- C ABI of the B200 (sm_100a) strongly-connected-component
 * engine.  Drop-in for iSpan's detection call.
 *
 * Reference interface replaced (paths inside the iSpan tree):
 *   void scc_detection(const graph *g, int alpha, int beta, int gamma,
 *                      double theta, index_t thread_count, double *avg_time)
 *       src/scc_common.h:15-23, defined at src/scc_core.cpp:27-1094
 *   void get_scc_result(index_t *scc_id, index_t vert_count)
 *       src/scc_common.h:25-28 (link-time hook, src/load_print.cpp:24-60)
 *   class graph {fw_beg_pos, fw_csr, bw_beg_pos, bw_csr, vert_count,
 *                edge_count}   src/graph.h:9-31, loaded by src/graph.cpp:2-92
 *
 * Plain pointers and sizes only.  Every call returns ISPAN_OK (0) or a
 * negative ISPAN_ERR_* code; nothing exits the process (the reference's
 * loader exits or asserts, src/graph.cpp:18-26).
 */
#ifndef ISPAN_B200_H
#define ISPAN_B200_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define ISPAN_OK 0
#define ISPAN_ERR_ARG (-1)       /* bad argument or malformed CSR */
#define ISPAN_ERR_NOMEM (-2)     /* device allocation or HBM budget exceeded */
#define ISPAN_ERR_CUDA (-3)      /* a CUDA runtime call failed */
#define ISPAN_ERR_TIMEOUT (-4)   /* a bounded device-side wait ran out */
#define ISPAN_ERR_INTERNAL (-5)  /* a device-side capacity check failed */
#define ISPAN_ERR_NODEV (-6)     /* no CUDA device / kernels not loadable */
#define ISPAN_ERR_CAPACITY (-7)  /* graph larger than the context was sized for */
#define ISPAN_ERR_BUSY (-8)      /* the server's request queue is full */

/* One directed graph in the reference's CSR layout (src/graph.h:9-31):
 * fw_beg/fw_adj = out-edges, bw_beg/bw_adj = in-edges (the transpose).
 * Offsets are int32 (the reference's width) or int64 (offset_bytes = 8),
 * vertex ids int32.  on_device = 1 when all four pointers are device memory
 * of the context's GPU; 0 when they are host memory (pinned memory uploads
 * fastest).  bw_beg and bw_adj both NULL: the forward CSR alone is given (and,
 * for host memory, copied); the scc runs build the reverse on the device,
 * which halves the bytes a host graph sends over PCIe.  Where about 9 bytes
 * an edge and 36 a vertex of scratch fit (kept by the context; copy chunks
 * below 2^31 edges), its lists are sorted chunk by chunk by a radix sort
 * (increasing source order); otherwise they are placed by atomics, in no
 * particular order.  ispan_scc_run_graphs needs both
 * directions. */
typedef struct {
    int64_t V, E;
    const void *fw_beg, *bw_beg;
    const int32_t *fw_adj, *bw_adj;
    int32_t offset_bytes;
    int32_t on_device;
} ispan_csr;

/* Direction-switch parameters of the reference's reachability searches
 * (src/fw_bw.h:576-624; CLI order of src/scc_main.cpp:16-25).  alpha: switch
 * top-down -> bottom-up when frontier edges exceed unexplored edges / alpha;
 * beta, gamma: switch bottom-up -> queue top-down when the frontier falls
 * below |worklist| / beta or the level exceeds gamma.  theta is the
 * reference's trim stop ratio; the peel here runs to a fixpoint, so theta is
 * accepted and recorded only.  Zero fields take the reference defaults
 * 30/200/10/0.1 (src/bash_one.sh:4). */
typedef struct {
    int32_t alpha, beta, gamma;
    double theta;
    uint32_t flags;
} ispan_params;

#define ISPAN_F_LABELS_ON_DEVICE 1u /* labels_out is device memory */
#define ISPAN_F_NO_GRAPH 2u         /* launch stages directly, no CUDA graph */
#define ISPAN_F_STAGE_TIMES 4u      /* record per-stage device times */
#define ISPAN_F_NO_L2_WINDOW 8u     /* no persisting L2 window over the status maps */
#define ISPAN_F_VALIDATE 16u        /* check a device-resident CSR before the run
                                       (host CSRs are always checked) */
#define ISPAN_F_EXACT_STATS 32u     /* also fill fw_edges / bw_edges and the trims' worklist
                                       sizes (extra passes) */
#define ISPAN_F_REVERSE_ATOMIC 64u  /* forward-only input: place the reverse lists by atomics
                                       (no sort scratch; slower) */

/* Stage-time slots follow the reference's avg_time[15] meanings
 * (src/scc_core.cpp:24-25, :1037-1053): 0 trim, 1 elephant SCC, 2 mice SCC,
 * 3 total, 4 trim size_1, 5 trim size_2, 6 pivot selection (fused with the
 * first trim-1 pass here), 7 FW, 8 BW, 9 WCC, 10 mice FW-BW, 13 trim size_3.
 * Finer slots without a reference counterpart: 11 colouring of the large
 * WCCs (part of 10), 12 second trim-1 peel, 14 residual worklist after the
 * pivot SCCs, 15 first trim-1 peel (12, 14, 15 are parts of 4).
 * Milliseconds of device time. */
typedef struct {
    double stage_ms[16];
    int64_t scc_count;        /* number of SCCs (no phantom vertex, unlike Q1) */
    int64_t giant_size;       /* vertices of the pivot SCC(s) */
    int64_t n_trim1, n_trim2, n_trim3; /* vertices labelled by each trim */
    int64_t n_mice_vertices, n_mice_scc, n_wcc;
    int64_t fw_size, fw_levels, bw_levels, residual, color_rounds, local_wcc, trim_rounds;
    int64_t fw_edges;         /* sum of out-degrees over the forward set F (ISPAN_F_EXACT_STATS) */
    int64_t bw_edges;         /* sum of in-degrees over the pivot SCC(s) S (ISPAN_F_EXACT_STATS) */
    /* sparse size histogram: pairs (hist_size[i], hist_count[i]) sorted by
     * size; the caller supplies the arrays (hist_cap entries) or NULLs */
    int64_t *hist_size, *hist_count;
    int64_t hist_cap, hist_n;
    /* worklists of the trims (ISPAN_F_EXACT_STATS): the peel's input is the
     * residual after the pivot SCCs (`residual` vertices, sum of their out-
     * plus in-degrees resid_edges); trim-2/3 read the peel's survivors */
    int64_t resid_edges;
    int64_t peeled_residual;       /* vertices left after the first peel */
    int64_t peeled_residual_edges; /* sum of their out- plus in-degrees */
} ispan_stats;

typedef struct ispan_ctx ispan_ctx;

/* A context owns device scratch for graphs up to max_V vertices / max_E
 * edges (per run) on one device, plus a CUDA stream (or the caller's stream
 * set with ispan_ctx_set_stream).  Contexts are independent; one context must
 * not be used by two host threads at once. */
int ispan_ctx_create(int device, int64_t max_V, int64_t max_E, ispan_ctx **out);
int ispan_ctx_destroy(ispan_ctx *ctx);
int ispan_ctx_set_stream(ispan_ctx *ctx, void *cuda_stream);
/* device bytes a context of this size holds (without uploaded graphs) */
int64_t ispan_ctx_bytes(int64_t max_V, int64_t max_E);

/* Launch tunables of a context, chosen per graph-shape class by the
 * autotuner (ispan_b200/autotune.py).  They change scheduling only, never
 * labels.  Zero fields take the defaults.  The reference's only knobs are
 * alpha/beta/gamma/theta (src/scc_main.cpp:16-25); these have no counterpart. */
typedef struct {
    int64_t async_v;          /* a search goes asynchronous below this many frontier vertices (65536) */
    int64_t async_e;          /* ... and this many frontier edges (262144) */
    int32_t async_deg;        /* an asynchronous CTA expands vertices up to this degree itself (16) */
    int32_t bfs_ctas_per_sm;  /* CTAs per SM of the persistent searches, at most the occupancy limit (2) */
    int32_t color_levels;     /* colouring large WCCs: a warp works up to 4 * color_levels chunks of 32
                                 frontier entries per grid round before handing the rest back (32) */
    int32_t color_pivots;     /* about this many pivots in the first colouring round; doubles per round (1024) */
    int32_t color_compact;    /* colour the large WCCs on a compact copy of their subgraph (dense ids,
                                 only their edges among themselves): 1 on, -1 off (0: default, on) */
    int32_t pair_searches;    /* run the forward and backward giant searches at the same time (the
                                 backward one over all active vertices; pivot SCC = both sets'
                                 intersection): 1 on, -1 off, 0 on for graphs of at most 2^20 vertices */
    int32_t tiny_residual;    /* solve a residual of at most 1024 vertices (and 4096 edges among them per
                                 direction) after the giant SCC in one CTA, skipping the later stage
                                 kernels: 1 on (0: default, off) */
    int32_t pdl;              /* launch each stage kernel that follows another plain kernel with
                                 programmatic dependent launch, so its launch overlaps the previous
                                 kernel's tail: -1 off (0: default, on) */
} ispan_tuning;

/* NULL restores the defaults; the next run re-captures its CUDA graph. */
int ispan_ctx_set_tuning(ispan_ctx *ctx, const ispan_tuning *t);
/* the values in effect (defaults filled in; bfs_ctas_per_sm 0 = occupancy limit) */
int ispan_ctx_get_tuning(ispan_ctx *ctx, ispan_tuning *t);

/* Detect the SCCs of g.  labels_out[V] receives, for every vertex, the
 * minimum vertex id of its SCC (host memory unless ISPAN_F_LABELS_ON_DEVICE).
 * Replaces scc_detection (src/scc_core.cpp:27); st may be NULL. */
int ispan_scc_run(ispan_ctx *ctx, const ispan_csr *g, const ispan_params *p,
                  int32_t *labels_out, ispan_stats *st);

/* Batched form: g is a disjoint union of nseg graphs whose vertex ranges are
 * [vbase[i], vbase[i+1]) (vbase host array of nseg+1 entries, vbase[0] = 0,
 * vbase[nseg] = V; edges never cross ranges).  Every graph gets its own pivot
 * and giant search; labels are global vertex ids (subtract vbase[i] for a
 * graph-local id).  One set of stage launches covers all graphs. */
int ispan_scc_run_batch(ispan_ctx *ctx, const ispan_csr *g, int32_t nseg, const int64_t *vbase,
                        const ispan_params *p, int32_t *labels_out, ispan_stats *st);

/* Batched form over separate graphs: gs[0..n) are independent CSRs, each on
 * the host or the device (its own on_device) with its own offset width.  They
 * are packed on the device into the context's union buffers (checked on the
 * way: offsets monotone from 0 to E, ids in [0, V), else ISPAN_ERR_ARG and no
 * stage runs), run as one disjoint union (ispan_scc_run_batch), and graph
 * i's labels -- local min ids, as ispan_scc_run on gs[i] alone -- are written
 * to labels_out[i] (host or device memory, told apart by address).  The sum
 * of the graphs' V and E must fit the context; st covers the whole batch.
 * The reference's counterpart is one scc_detection call per graph
 * (src/scc_core.cpp:27). */
int ispan_scc_run_graphs(ispan_ctx *ctx, const ispan_csr *gs, int32_t n, int32_t *const *labels_out,
                         const ispan_params *p, ispan_stats *st);

/* The two phases of ispan_scc_run_graphs, for callers that overlap them:
 * pack copies and checks the graphs into the context's union buffers (host
 * copies, then two short kernels on the context's stream); run executes the
 * pipeline on the packed union and writes the labels.  A server packs batch
 * k+1 on one context while batch k runs on another.  run must get the same
 * gs sizes as the pack before it, else ISPAN_ERR_ARG. */
int ispan_graphs_pack(ispan_ctx *ctx, const ispan_csr *gs, int32_t n);
int ispan_graphs_run(ispan_ctx *ctx, const ispan_csr *gs, int32_t n, int32_t *const *labels_out,
                     const ispan_params *p, ispan_stats *st);

/* ---- served form: continuous batching over a request queue ------------
 * No counterpart in the reference (one graph per process).  A server runs
 * n_slots lanes, each a context with its own CUDA stream and worker thread,
 * concurrently on one GPU.  A lane whose batch is done takes its share of
 * the queued requests (arrival order) at once, while the other lanes'
 * batches are still running, so a request that arrives while others are on
 * the GPU is admitted as soon as a lane and memory free up and its work
 * overlaps theirs on the device.  Memory: the budget is one device
 * allocation made at creation; each batch's exact footprint (pipeline
 * scratch, union CSR and tables for its vertex, edge and graph counts) is
 * taken from it when the batch is admitted and returned when its labels are
 * written; a batch that does not fit the free memory waits.  A request's
 * graph and label buffer must stay valid until the request is reported
 * done. */
typedef struct ispan_server ispan_server;

typedef struct {
    int32_t device;
    int32_t max_batch_graphs;   /* graphs per batch; 0: 4096 */
    int32_t n_slots;            /* lanes running batches concurrently; 0: 4.  With
                                   more than one, each lane's persistent stages use
                                   0.9 / n_slots of the SMs */
    int32_t reserved;
    int64_t hbm_budget_bytes;   /* device memory the server holds (allocated at
                                   creation); 0: 64 GiB */
    int64_t max_batch_V;        /* vertices / edges of a batch of several graphs (0: no */
    int64_t max_batch_E;        /*   limit but the footprint one).  A batch of several
                                   graphs takes at most half the budget (the whole budget
                                   with one lane); a single larger request runs alone if its
                                   footprint fits the budget */
    int64_t max_wait_us;        /* a partial batch waits this long for more requests */
    int64_t max_pending;        /* queued requests before submit returns ISPAN_ERR_BUSY; 0: no limit */
    ispan_params params;
} ispan_server_config;

typedef struct {
    int32_t status;          /* 0 queued or running, 1 done, or an ISPAN_ERR_* code */
    int32_t batch_graphs;    /* graphs in the batch that served it */
    int64_t batch_id;
    int64_t t_submit_ns;     /* CLOCK_MONOTONIC */
    int64_t t_start_ns;      /* its batch was admitted (set while it runs) */
    int64_t t_done_ns;       /* its labels were written */
} ispan_request_info;

/* Fails with ISPAN_ERR_NOMEM when the budget cannot be allocated or the
 * explicit batch size does not fit it. */
int ispan_server_create(const ispan_server_config *cfg, ispan_server **out);
int ispan_server_limits(const ispan_server *s, int64_t *max_V, int64_t *max_E, int32_t *max_graphs);
/* Queue one graph (host or device CSR); labels_out[g->V] (host or device)
 * receives its local min-id labels.  A graph whose footprint exceeds the
 * whole budget is refused with ISPAN_ERR_CAPACITY. */
int ispan_server_submit(ispan_server *s, const ispan_csr *g, int32_t *labels_out, int64_t *ticket);
/* 1 done, 0 not yet, or the request's error; a finished request is reported
 * once (a second poll of its ticket returns ISPAN_ERR_ARG). */
int ispan_server_poll(ispan_server *s, int64_t ticket, ispan_request_info *info);
/* As poll, blocking up to timeout_us (negative: no limit); 0 on timeout. */
int ispan_server_wait(ispan_server *s, int64_t ticket, int64_t timeout_us, ispan_request_info *info);
/* Up to n of: batches, graphs, vertices, edges served; busy ns (wall time
 * with at least one batch in flight); queued requests; lane ns (sum of the
 * batches' wall times: lane ns / busy ns is the mean number of batches in
 * flight); budget bytes in use; peak budget bytes in use; lanes. */
int ispan_server_counters(ispan_server *s, int64_t *out, int32_t n);
/* Serves what is queued, then stops the lanes and frees the device memory. */
int ispan_server_destroy(ispan_server *s);

/* Condensation: the DAG of the SCCs of a device-resident graph g (only its
 * forward CSR is read) given device labels[V] from a run on it.  Components
 * are named by their canonical labels; pairs_out (host or device, up to cap
 * entries) receives each distinct crossing pair as (source label << 32 |
 * target label), sorted; *n_pairs gets the number of distinct pairs (call
 * with cap 0 to size the buffer).  Allocates temporary device memory.  The
 * reference stops at class counts (src/load_print.cpp:24-60); this is the
 * step after the path. */
int ispan_condense(const ispan_csr *g, const int32_t *labels, uint64_t *pairs_out, int64_t cap,
                   int64_t *n_pairs, void *stream);

/* One rank's level of a reachability search over a graph whose rows are
 * split across GPUs: rows holds the CSR rows of the vertices [v0, v0 +
 * rows->V) (forward rows for a forward search, backward rows for a backward
 * one; fw_beg/fw_adj are read, offsets local, adjacency global ids, device
 * memory).  Every owned vertex set in frontier[] (byte per vertex, V
 * entries) marks next[w] = 1 for each neighbour w not in visited[] and, if
 * allowed is not NULL, set in allowed[].  The caller merges the ranks' next
 * maps with a MAX all-reduce (ispan_b200/sharded.py).  Replaces the per-level
 * step of the reference's MPI variant (src_mpi/fw_bw.h:382-442). */
int ispan_shard_expand(const ispan_csr *rows, int64_t v0, int64_t V, const uint8_t *frontier,
                       const uint8_t *visited, const uint8_t *allowed, uint8_t *next, void *stream);

/* Queue form of a sharded level (what ispan_b200/sharded.py runs).
 * expand_queue: the owned frontier vertices queue[0 .. *queue_count) (global
 * ids; the count is read on the device) mark next[w] = 1 (byte per vertex, V
 * entries) for each neighbour w whose bit is clear in visited[] and, if
 * allowed is not NULL, set in allowed[] (both bitmaps of V bits, replicated
 * on every rank).  collect: after the ranks' next maps are merged by a
 * reduce-scatter (MAX) that leaves this rank its owned slice mine[0 .. n_own)
 * of the vertices [v0, v0 + n_own) (v0 a multiple of 32), the owned vertices
 * set there and not yet visited get their visited bit and are appended to
 * queue (count *queue_count, which the caller zeroes first); the caller then
 * all-gathers the owned visited words.  Replaces the per-level step of the
 * reference's MPI variant with its bitmap exchange (src_mpi/fw_bw.h:382-442). */
int ispan_shard_expand_queue(const ispan_csr *rows, int64_t v0, int64_t V, const int32_t *queue,
                             const int64_t *queue_count, const uint32_t *visited, const uint32_t *allowed,
                             uint8_t *next, void *stream);
int ispan_shard_collect(int64_t v0, int64_t n_own, const uint8_t *mine, uint32_t *visited, int32_t *queue,
                        int64_t *queue_count, void *stream);

/* Largest graph (vertices) that ispan_scc_small_noalloc accepts. */
#define ISPAN_NOALLOC_MAX_V 65536

/* SCC labels of one small graph without allocating any device memory.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * code running under another framework's memory manager (which owns the
 * device memory), latency-critical paths that cannot take cudaMalloc's
 * implicit synchronisation, or code issuing work during stream capture.
 * g must be device-resident (on_device = 1; only the forward CSR is read);
 * labels_out is device memory of V entries and receives the same canonical
 * min-id labels as ispan_scc_run.  The work is one kernel launched on
 * `stream` (NULL: the default stream); the call returns once it is queued.
 * Scratch is a fixed 2 MiB device array inside the library, so graphs above
 * ISPAN_NOALLOC_MAX_V vertices are rejected with ISPAN_ERR_CAPACITY.  Every
 * device that loads the library holds that array until the process exits.
 * The first call on a device resolves the array's address (no allocation);
 * make that first call before any stream capture.  All calls on a device
 * share the one array: calls that overlap on the GPU (different streams,
 * no ordering between them) race and must not be issued.  The kernel checks
 * the graph before using any index read from it (offsets monotone from 0 to
 * E, every id in [0, V)); a malformed graph gets -1 in every label (valid
 * labels are never negative) and nothing past its arrays is touched.  An
 * error already pending on the calling thread is returned as ISPAN_ERR_CUDA
 * without clearing it and without a launch. */
int ispan_scc_small_noalloc(const ispan_csr *g, int32_t *labels_out, void *stream);

/* Reference-convention per-vertex codes from canonical labels and the class
 * of each vertex, as get_scc_result (src/load_print.cpp:24-60) expects:
 * 1 giant, -1 trimmed size-1, -2 size-2, -3 size-3, otherwise label + 2;
 * codes_out has V+1 entries, the last (the reference's phantom slot) 0.
 * Valid after the most recent run on ctx; host memory. */
int ispan_ref_codes(ispan_ctx *ctx, int32_t *codes_out);

/* Diagnostics: per-level trace of the two reachability searches of the last
 * run, [4][256][4] int64: for the forward (0) and backward (1) search, per
 * level, mode (0 top-down, 1 bottom-up, 2 asynchronous), vertices reached,
 * frontier edges, %globaltimer ns; for the large-WCC rounds (2), per round,
 * round number (bits 0-15; grid-wide rounds of its forward search in bits
 * 16-39, of its backward search from bit 40), vertices left, pivots,
 * %globaltimer ns; and (3), for a run with ISPAN_F_EXACT_STATS, per round,
 * its forward relaxation's pops, edges checked, vertices queued and ns that
 * warps waited for work, each summed over all warps.
 * No counterpart in the reference (its VERBOSE "Level-k" lines, src/fw_bw.h:557-572,
 * print the same kind of record). */
int ispan_debug_trace(ispan_ctx *ctx, int64_t *out, int64_t cap);

/* Failure detection, exercised without a GPU fault: runs the persistent
 * stages' bounded grid barrier with a CTA that never arrives and a limit of
 * limit_us (at most 10 s); the waiting CTA gives up, records
 * ISPAN_ERR_TIMEOUT and returns, which this call returns.  The context stays
 * usable.  No counterpart in the reference (it has no bounded waits). */
int ispan_debug_barrier_timeout(ispan_ctx *ctx, int64_t limit_us);

const char *ispan_strerror(int code);
/* library version string */
const char *ispan_version(void);

#ifdef __cplusplus
}
#endif
#endif

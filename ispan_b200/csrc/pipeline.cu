// pipeline.cu -- host side of the B200 SCC engine: contexts, device memory,
// the stage launch sequence (captured once into a CUDA graph and replayed),
// and the extern "C" boundary declared in include/ispan_b200.h.
//
// Stage sequence (reference src/scc_core.cpp:144-1070, same order):
//   trim-1-first + pivot      k_trim1_first, k_seed
//   elephant FW / BW          k_bfs<.,0>, k_bfs<.,1>   (persistent, cooperative)
//   giant, residual           k_giant_residual
//   trim-1 peel (fixpoint)    k_trim1                  (persistent, cooperative)
//   trim-2, trim-3            k_trim2, k_trim3
//   trim-1 peel again         k_trim1
//   WCC                       k_wcc_init/hook/compress/giant/hook/flatten/alloc/scatter
//   mice: small WCCs          k_local_scc              (shared-memory Tarjan)
//   mice: large WCCs          k_color                  (persistent, cooperative)
//   canonical labels          k_finalize
// Every kernel reads its work sizes from device memory, so the whole sequence
// is enqueued without a host round trip and the host synchronises once.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "bfs.cuh"
#include "pack.cuh"
#include "transpose.cuh"
#include "compact.cuh"
#include "tiny.cuh"
#include "lane.h"
#include "stages.cuh"

using namespace ispan;

namespace {

#define CK(x)                                                                        \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess) {                                                     \
            fprintf(stderr, "ispan_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(e_), \
                    __FILE__, __LINE__);                                             \
            return ISPAN_ERR_CUDA;                                                   \
        }                                                                            \
    } while (0)

// A context's scratch comes from cudaMalloc, or -- for a server lane -- is
// carved out of a region of the server's device-memory budget.  A region
// with a null base only measures (the footprint of a carve).
struct Region {
    char *base = nullptr;
    size_t cap = 0, used = 0;
};

template <typename T>
static int dalloc(T **p, size_t n, std::vector<void *> &owned, Region *rg = nullptr) {
    if (n == 0) n = 1;
    if (rg) {
        const size_t at = (rg->used + 255) / 256 * 256, bytes = n * sizeof(T);
        if (rg->base && at + bytes > rg->cap) return ISPAN_ERR_NOMEM;
        *p = rg->base ? (T *)(rg->base + at) : nullptr;
        rg->used = at + bytes;
        return ISPAN_OK;
    }
    void *q = nullptr;
    if (cudaMalloc(&q, n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return ISPAN_ERR_NOMEM;
    }
    owned.push_back(q);
    *p = (T *)q;
    return ISPAN_OK;
}

// Failure-detection probe: a two-CTA grid whose second CTA never reaches
// the barrier, so the first waits in grid_sync until its time limit, sets
// the error word and returns (the same bounded wait every persistent stage
// uses, with a short limit).
__global__ void k_barrier_probe(unsigned *gs, int *err, uint64_t limit_ns) {
    if (blockIdx.x == 1) return;  // this CTA never arrives
    grid_sync(gs, err, limit_ns);
}

constexpr int kNumEv = 13;  // stage boundaries recorded per run
constexpr int kUpChunks = 8;  // forward adjacency copied in chunks, each counted as it lands

}  // namespace

struct ispan_ctx {
    int device = 0;
    int nsm = 148;
    int nsm_coop = 0;               // SMs the persistent grids are sized for (0: all)
    Region *rg = nullptr;           // scratch carved from a server's budget (lanes)
    Region lane_region;             // the region rg points to while a lane is bound
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int64_t maxV = 0, maxE = 0, maxW = 0;
    int64_t maxSeg = 0;
    std::vector<void *> owned;      // fixed scratch
    std::vector<void *> seg_owned;  // per-segment arrays (grow on demand)
    std::vector<void *> csr_owned;  // uploaded host graphs

    // device scratch
    int32_t *label = nullptr;
    uint8_t *cls = nullptr;
    uint32_t *A = nullptr, *F = nullptr, *B = nullptr, *D = nullptr, *P = nullptr, *T = nullptr;
    uint32_t *bits = nullptr;  // the block holding A..T
    int64_t bits_bytes = 0;
    bool l2_limit_set = false;

    // union buffers of ispan_scc_run_graphs (allocated on first use)
    int64_t *pk_fwb = nullptr, *pk_bwb = nullptr;  // [maxV + 1]
    int32_t *pk_fwa = nullptr, *pk_bwa = nullptr;  // [maxE]
    int64_t *pk_stage = nullptr;                   // staged host offsets [2 * (stage_V + pk_n)]
    int64_t stage_V = -1;                          // vertices of host graphs a batch may stage (-1: maxV)
    PackDesc *pk_desc = nullptr;                   // [pk_n]
    int64_t *pk_vb = nullptr, *pk_eb = nullptr;    // [pk_n + 1]
    PackDesc *h_desc = nullptr;                    // pinned mirrors
    int64_t *h_vbeb = nullptr;                     // pinned [2 * (pk_n + 1)]
    int64_t pk_n = 0;
    int64_t h_cap = 0;                             // entries of the pinned mirrors
    std::vector<void *> pk_owned;                  // union buffers
    std::vector<void *> pkt_owned;                 // per-graph tables
    std::vector<int64_t> pk_vbase;  // segmentation of the packed union
    int64_t pk_cur_n = 0, pk_Et = 0;
    bool pk_ready = false;          // a packed union waits for its run
    int32_t *qv[2] = {nullptr, nullptr};
    int64_t *qe[2] = {nullptr, nullptr};
    int32_t *qchunk[2] = {nullptr, nullptr};
    int32_t *wl[2] = {nullptr, nullptr};
    int32_t *wl4 = nullptr;  // wl[0], wl[1], members, roots: one block of 4 x (maxV + 32)
    int32_t *cnt_out = nullptr, *cnt_in = nullptr, *parent = nullptr, *aux = nullptr, *aux2 = nullptr,
            *members = nullptr, *roots = nullptr, *small = nullptr, *large[2] = {nullptr, nullptr};
    unsigned long long *ctlblk = nullptr;  // counters | qpk | lvl | ctl64
    int64_t *hist = nullptr;
    unsigned int *gsync = nullptr;
    int *err = nullptr;
    BfsCtl *bfsctl = nullptr;
    long long *trace = nullptr;
    int64_t *vbase = nullptr;
    unsigned long long *pivot_key = nullptr, *gsize = nullptr;
    int32_t *gmin = nullptr;

    // uploaded CSR (host input), and the reverse CSR built on the device
    // for input that gives the forward direction only
    void *up_fw_beg = nullptr, *up_bw_beg = nullptr;
    int32_t *up_fw_adj = nullptr, *up_bw_adj = nullptr;
    int64_t up_V = -1, up_E = -1;
    cudaEvent_t ev_up[kUpChunks] = {};  // forward adjacency chunk k copied
    void *scan_tmp = nullptr;           // the reverse offsets' scan
    size_t scan_tmp_bytes = 0;
    // the reverse lists by a radix sort of (id, source) pairs, chunk by
    // chunk: keys and sources of all edges, a chunk's alternates, the
    // running in-degree counts after each chunk, a chunk's run starts, and
    // the sort's and scan's temporary storage
    int32_t *rv_k0 = nullptr, *rv_v = nullptr, *rv_k1 = nullptr, *rv_v1 = nullptr;
    int32_t *rv_snap = nullptr, *rv_run = nullptr;
    void *rv_tmp = nullptr;
    size_t rv_tmp_bytes = 0;
    int64_t rv_E = -1, rv_V = -1;
    bool rv_failed = false;  // the scratch did not fit: placement by atomics
    std::vector<void *> rv_owned;

    // host staging
    unsigned long long *h_counters = nullptr;  // pinned
    int *h_err = nullptr;

    ispan_tuning tuning = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};

    // launch geometry
    int g_stream = 0;           // grid for plain grid-stride kernels
    int g_coop[5] = {0, 0, 0, 0, 0};  // bfs<0>, bfs<1>, trim1, color, color on the compact graph
    int g_pair = 0;             // each search's grid when the two run at the same time

    // the backward search's stream when the searches run at the same time
    cudaStream_t stream2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int g_coop_w = 0;           // offset width the coop grids were computed for

    // CUDA graph cache
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // without / with the stage-time events
    char gkey[2][256];
    bool graph_broken = false;
    cudaEvent_t ev[kNumEv];
    bool have_ev = false;

    // last run (for ispan_ref_codes)
    int64_t last_V = 0;
    int32_t *last_label = nullptr;
    int64_t last_nseg = 1;
    std::vector<int64_t> vbase_host;  // segmentation currently on the device
    bool validate_next = false;       // an uploaded host CSR is checked once on the device
    std::mutex mu;
};

static int64_t words_of(int64_t V) { return (V + 31) / 32 + 1; }

// the cached CUDA graphs hold pointers and launch shapes: dropped whenever those change
static void drop_graphs(ispan_ctx *c) {
    for (int i = 0; i < 2; ++i)
        if (c->gexec[i]) {
            cudaGraphExecDestroy(c->gexec[i]);
            c->gexec[i] = nullptr;
        }
}

static constexpr int64_t kL2WindowMinBytes = 4 << 20;  // status maps smaller than this get no L2 window
static constexpr int kCtlCounters = 0;                       // kNumCounters
static constexpr int kCtlQpk = kNumCounters;                 // 3 (forward search)
static constexpr int kCtlLvl = kNumCounters + 4;             // 12
static constexpr int kCtlX = kNumCounters + 4 + 16;          // kNumCtl
static constexpr int kCtlQpkB = kCtlX + kNumCtl;             // 3 (backward search: fresh slots,
static constexpr int kCtlLvlB = kCtlQpkB + 4;                //    no reset between the searches)
static constexpr int kCtlTotal = kCtlLvlB + 16;

extern "C" int64_t ispan_ctx_bytes(int64_t V, int64_t E) {
    int64_t W = words_of(V);
    int64_t b = 0;
    b += V * 4 + V;                 // label, cls
    b += 6 * ((W + 63) / 64 * 64) * 4;  // bitmaps
    b += 2 * (V * 4 + (V + 1) * 8); // queues
    b += 2 * ((E / kChunk + 4) * 4);
    b += 2 * V * 4;                 // worklists
    b += 10 * V * 4;                // counters, parent, aux, aux2, members, roots, small, large x2
    b += (kHistCap + kBigCap) * 8;
    return b;
}

static int ctx_alloc(ispan_ctx *c) {
    int64_t V = c->maxV + 32, E = c->maxE;
    int64_t W = words_of(V);
    c->maxW = W;
    int rc = 0;
    auto &o = c->owned;
    Region *g = c->rg;
    rc |= dalloc(&c->label, V, o, g);
    rc |= dalloc(&c->cls, V, o, g);
    // the six status maps in one block, so one L2 access-policy window covers them
    const int64_t Wp = (W + 63) / 64 * 64;  // 256-byte aligned slices
    rc |= dalloc(&c->bits, 6 * Wp, o, g);
    c->bits_bytes = 6 * Wp * 4;
    if (!rc) {
        c->A = c->bits;
        c->F = c->bits + Wp;
        c->B = c->bits + 2 * Wp;
        c->D = c->bits + 3 * Wp;
        c->P = c->bits + 4 * Wp;
        c->T = c->bits + 5 * Wp;
    }
    for (int i = 0; i < 2; ++i) {
        rc |= dalloc(&c->qv[i], V, o, g);
        rc |= dalloc(&c->qe[i], V + 1, o, g);
        rc |= dalloc(&c->qchunk[i], E / kChunk + 4, o, g);

        rc |= dalloc(&c->large[i], V, o, g);
    }
    rc |= dalloc(&c->cnt_out, V, o, g);
    rc |= dalloc(&c->cnt_in, V, o, g);
    rc |= dalloc(&c->parent, V, o, g);
    rc |= dalloc(&c->aux, V, o, g);
    rc |= dalloc(&c->aux2, V, o, g);
    // the two worklists, then the WCC member and root lists, in one block:
    // the compact colouring graph (compact.cuh) uses the first two as one
    // out-adjacency array of 2 V entries and the last two as the in-adjacency
    rc |= dalloc(&c->wl4, 4 * V, o, g);
    if (!rc) {
        c->wl[0] = c->wl4;
        c->wl[1] = c->wl4 + V;
        c->members = c->wl4 + 2 * V;
        c->roots = c->wl4 + 3 * V;
    }
    rc |= dalloc(&c->small, V, o, g);
    rc |= dalloc(&c->ctlblk, kCtlTotal, o, g);
    rc |= dalloc(&c->hist, kHistCap + kBigCap, o, g);
    rc |= dalloc(&c->gsync, 2 * kGridSyncWords, o, g);  // the second block: a backward search run beside
    rc |= dalloc(&c->err, 4, o, g);
    rc |= dalloc(&c->bfsctl, 1, o, g);
    rc |= dalloc(&c->trace, 4 * kTraceLevels * 4, o, g);
    return rc ? ISPAN_ERR_NOMEM : ISPAN_OK;
}

static int ctx_segments(ispan_ctx *c, int64_t nseg) {
    if (nseg <= c->maxSeg) return ISPAN_OK;
    if (c->rg && c->maxSeg > 0) return ISPAN_ERR_CAPACITY;  // a lane's tables were carved for its batch
    if (!c->rg) {  // a lane frees nothing (cudaFree would synchronise the device); destroy frees these
        for (void *p : c->seg_owned) cudaFree(p);
        c->seg_owned.clear();
    }
    int64_t n = std::max<int64_t>(nseg, 1);
    int rc = 0;
    rc |= dalloc(&c->vbase, n + 1, c->seg_owned, c->rg);
    rc |= dalloc(&c->pivot_key, n, c->seg_owned, c->rg);
    rc |= dalloc(&c->gsize, n, c->seg_owned, c->rg);
    rc |= dalloc(&c->gmin, n, c->seg_owned, c->rg);
    if (rc) {
        c->maxSeg = 0;
        return ISPAN_ERR_NOMEM;
    }
    c->maxSeg = n;
    drop_graphs(c);
    c->vbase_host.clear();
    return ISPAN_OK;
}

template <typename K>
static int coop_grid(K kernel, int nsm, int block) {
    int per = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, block, 0) != cudaSuccess || per < 1) {
        cudaGetLastError();
        return 0;
    }
    return per * nsm;
}

template <typename OffT>
static void fill_run(ispan_ctx *c, Run<OffT> &r, Ext<OffT> &x, int64_t V, int64_t E, int32_t nseg,
                     const OffT *fwb, const OffT *bwb, const int32_t *fwa, const int32_t *bwa, int32_t *label,
                     const ispan_params *p) {
    r.V = V;
    r.E = E;
    r.W = (V + 31) / 32;
    r.nseg = nseg;
    r.vbase = c->vbase;
    r.fw_beg = fwb;
    r.bw_beg = bwb;
    r.fw_adj = fwa;
    r.bw_adj = bwa;
    r.label = label;
    r.A = c->A; r.F = c->F; r.B = c->B; r.D = c->D; r.P = c->P; r.T = c->T;
    for (int i = 0; i < 2; ++i) {
        r.qv[i] = c->qv[i];
        r.qe[i] = c->qe[i];
        r.qchunk[i] = c->qchunk[i];
        r.wl[i] = c->wl[i];
    }
    r.qpk = c->ctlblk + kCtlQpk;
    r.lvl = c->ctlblk + kCtlLvl;
    r.wlc = nullptr;
    r.cnt_out = c->cnt_out;
    r.cnt_in = c->cnt_in;
    r.parent = c->parent;
    r.aux = c->aux;
    r.aux2 = c->aux2;
    r.members = c->members;
    r.pivot_key = c->pivot_key;
    r.gmin = c->gmin;
    r.gsize = c->gsize;
    r.cls = c->cls;
    r.counters = c->ctlblk + kCtlCounters;
    r.hist = c->hist;
    r.gsync = c->gsync;
    r.err = c->err;
    r.trace = c->trace;
    r.alpha = p && p->alpha > 0 ? p->alpha : 30;
    r.beta = p && p->beta > 0 ? p->beta : 200;
    r.gamma = p && p->gamma > 0 ? p->gamma : 10;
    r.flags = (p ? p->flags : 0) & ~kRunPair;  // set by enqueue when the searches run together
    r.async_v = c->tuning.async_v > 0 ? c->tuning.async_v : kAsyncV;
    r.async_e = c->tuning.async_e > 0 ? c->tuning.async_e : kAsyncE;
    r.async_deg = c->tuning.async_deg > 0 ? c->tuning.async_deg : kAsyncDeg;
    r.color_levels = c->tuning.color_levels > 0 ? c->tuning.color_levels : kCLevels;
    r.color_pivots = c->tuning.color_pivots > 0 ? c->tuning.color_pivots : kCPivots;
    x.ctl = c->ctlblk + kCtlX;
    x.roots = c->roots;
    x.small = c->small;
    x.large[0] = c->large[0];
    x.large[1] = c->large[1];
    x.cq[0] = c->qv[0];  // the frontier queues are free once the giant is done
    x.cq[1] = c->qv[1];
    x.cand = c->small;   // free until the WCC stage lists its small components
}

// The run descriptor of the colouring on the compact graph: the same state
// arrays, the compact CSR (int32 offsets) and the compact-to-original map.
template <typename OffT>
static void compact_run(const Run<OffT> &r, const Ext<OffT> &x, const CmpBufs &b, Run<int32_t> &rc,
                        Ext<int32_t> &xc) {
    memset(&rc, 0, sizeof rc);
    memset(&xc, 0, sizeof xc);
    rc.V = r.V;  // an upper bound: the compact vertex count is read on the device
    rc.E = r.E;
    rc.W = r.W;
    rc.nseg = r.nseg;
    rc.vbase = r.vbase;
    rc.fw_beg = b.fbeg;
    rc.bw_beg = b.bbeg;
    rc.fw_adj = b.fadj;
    rc.bw_adj = b.badj;
    rc.label = r.label;
    rc.A = r.A; rc.F = r.F; rc.B = r.B; rc.D = r.D; rc.P = r.P; rc.T = r.T;
    for (int i = 0; i < 2; ++i) {
        rc.qv[i] = r.qv[i];
        rc.qe[i] = r.qe[i];
        rc.qchunk[i] = r.qchunk[i];
        rc.wl[i] = r.wl[i];
    }
    rc.qpk = r.qpk;
    rc.lvl = r.lvl;
    rc.wlc = r.wlc;
    rc.cnt_out = r.cnt_out;
    rc.cnt_in = r.cnt_in;
    rc.parent = r.parent;
    rc.aux = r.aux;
    rc.aux2 = r.aux2;
    rc.members = r.members;
    rc.pivot_key = r.pivot_key;
    rc.gmin = r.gmin;
    rc.gsize = r.gsize;
    rc.cls = r.cls;
    rc.counters = r.counters;
    rc.hist = r.hist;
    rc.gsync = r.gsync;
    rc.trace = r.trace;
    rc.err = r.err;
    rc.alpha = r.alpha;
    rc.beta = r.beta;
    rc.gamma = r.gamma;
    rc.flags = r.flags;
    rc.async_v = r.async_v;
    rc.async_e = r.async_e;
    rc.async_deg = r.async_deg;
    rc.color_levels = r.color_levels;
    rc.color_pivots = r.color_pivots;
    xc.ctl = x.ctl;
    xc.roots = x.roots;
    xc.small = x.small;
    xc.large[0] = x.large[0];
    xc.large[1] = x.large[1];
    xc.cq[0] = x.cq[0];
    xc.cq[1] = x.cq[1];
    xc.cand = x.cand;
    xc.old = b.old;
}

// A plain launch, with programmatic stream serialization when pdl is set.
template <typename... P, typename... A>
static cudaError_t launch_k(bool pdl, void (*k)(P...), int64_t grid, int block, cudaStream_t s, A... args) {
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.stream = s;
    cudaLaunchAttribute at;
    memset(&at, 0, sizeof at);
    at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at.val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = &at;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, args...);
}

template <typename Kern, typename... Args>
static cudaError_t launch_coop(Kern k, int grid, cudaStream_t s, Args... args) {
    void *ptrs[] = {(void *)&args...};
    return cudaLaunchCooperativeKernel((const void *)k, dim3(grid), dim3(kBlock), ptrs, 0, s);
}

// Whether the two searches of a run go at the same time.  On a small graph
// each search level costs a few microseconds of dependent loads and a grid
// barrier whatever its work, so running the backward search beside the
// forward one (over the active map, pivot SCC = F & B) halves the levels in
// sequence; on a large graph the backward search inside F does less work.
// The backward search then takes buffers that are free until the giant is
// done: the colouring lists as its vertex queues, the worklist block as its
// edge prefixes, the peel counters as its chunk maps, D for its snapshots.
template <typename OffT>
static bool pair_searches(const ispan_ctx *c, const Run<OffT> &r) {
    const int t = c->tuning.pair_searches;
    if (t < 0 || !c->stream2 || c->g_pair < 1) return false;
    if (r.E / kChunk + 4 > c->maxV + 32) return false;  // chunk maps must fit the peel counters
    return t > 0 || r.V <= kPairMaxV;
}

// Enqueue the whole pipeline on c->stream (plain launches; may be captured).
template <typename OffT>
static cudaError_t enqueue(ispan_ctx *c, Run<OffT> r, Ext<OffT> x, bool times, bool capturing) {
    cudaStream_t s = c->stream;
    const int G = c->g_stream;
    unsigned long long *ctl = c->ctlblk;
    cudaError_t e;
    const bool pair = pair_searches(c, r);
    if (pair) r.flags |= kRunPair;
    // a plain kernel that directly follows another plain kernel on s is
    // launched for programmatic dependent launch (see pdl_wait); after an
    // event or a cooperative launch the ordinary stream order applies
    bool prev_plain = false;
    const bool pdl_ok = c->tuning.pdl >= 0;
#define EV(i) \
    if (times) { e = cudaEventRecordWithFlags(c->ev[i], s, capturing ? cudaEventRecordExternal : 0); if (e) return e; prev_plain = false; }
#define LK(...) \
    do { __VA_ARGS__; e = cudaGetLastError(); if (e) return e; } while (0)
#define PK(kern, grid, block, ...) \
    do { e = launch_k(pdl_ok && prev_plain, kern, (grid), (block), s, __VA_ARGS__); if (e) return e; prev_plain = true; } while (0)
    EV(0);
    {   // every per-run counter, map and table that starts at zero, in one launch
        ResetDesc rd;
        rd.z[0] = {ctl, (int64_t)kCtlTotal * 8};
        rd.z[1] = {c->hist, (int64_t)(kHistCap + kBigCap) * 8};
        rd.z[2] = {c->gsync, 2 * kGridSyncWords * 4};
        rd.z[3] = {c->err, 4 * 4};
        rd.z[4] = {c->trace, 4 * kTraceLevels * 4 * 8};
        rd.z[5] = {c->pivot_key, r.nseg * 8};
        rd.z[6] = {c->gsize, r.nseg * 8};
        rd.gmin = c->gmin;
        rd.nseg = r.nseg;
        PK((k_reset), std::min<int64_t>(G, 4 * c->nsm), 256, rd);
    }
    PK((k_trim1_first<OffT>), G, kBlock, r, x);
    EV(1);
    const int gseed = (int)std::max<int64_t>(1, (r.nseg + 1023) / 1024);
    Run<OffT> rb = r;  // the backward search counts in its own queue and level slots
    rb.qpk = ctl + kCtlQpkB;
    rb.lvl = ctl + kCtlLvlB;
    if (pair) {
        const int64_t Vp = c->maxV + 32;  // entries of each scratch array
        rb.qv[0] = c->large[0];
        rb.qv[1] = c->large[1];
        rb.qe[0] = reinterpret_cast<int64_t *>(c->wl4);
        rb.qe[1] = reinterpret_cast<int64_t *>(c->wl4 + 2 * Vp);
        rb.qchunk[0] = c->cnt_out;
        rb.qchunk[1] = c->cnt_in;
        rb.P = c->D;
        rb.gsync = c->gsync + kGridSyncWords;
        PK((k_seed<OffT, 0>), gseed, 32 * 32, r);
        PK((k_seed<OffT, 1>), gseed, 32 * 32, rb);
        if ((e = cudaEventRecord(c->ev_fork, s))) return e;
        prev_plain = false;
        if ((e = cudaStreamWaitEvent(c->stream2, c->ev_fork, 0))) return e;
        if ((e = launch_coop(k_bfs<OffT, 1>, c->g_pair, c->stream2, rb, c->bfsctl))) return e;
        prev_plain = false;
        if ((e = launch_coop(k_bfs<OffT, 0>, c->g_pair, s, r, c->bfsctl))) return e;
        prev_plain = false;
        EV(2);
        if ((e = cudaEventRecord(c->ev_join, c->stream2))) return e;
        if ((e = cudaStreamWaitEvent(s, c->ev_join, 0))) return e;
        prev_plain = false;
    } else {
        PK((k_seed<OffT, 0>), gseed, 32 * 32, r);
        if ((e = launch_coop(k_bfs<OffT, 0>, c->g_coop[0], s, r, c->bfsctl))) return e;
        prev_plain = false;
        EV(2);
        PK((k_seed<OffT, 1>), gseed, 32 * 32, rb);
        if ((e = launch_coop(k_bfs<OffT, 1>, c->g_coop[1], s, rb, c->bfsctl))) return e;
        prev_plain = false;
    }
    if (r.flags & ISPAN_F_EXACT_STATS) PK((k_reach_degrees<OffT>), G, kBlock, r);
    EV(3);
    PK((k_giant_residual<OffT>), G, kBlock, r, x);
    if (r.flags & ISPAN_F_EXACT_STATS) PK((k_list_degrees<OffT>), G, kBlock, r, r.wl[0], x.ctl + K_WL0, -1, C_Q1_XDEG);
    EV(4);
    // on request, a residual of at most kTinyV vertices is solved here in
    // one CTA, and every stage kernel up to the finalisation then returns at
    // once (off by default: on R-MAT graphs the residual holds hubs whose
    // lists one CTA scans slower than the stage kernels' full grids)
    if (c->tuning.tiny_residual > 0) PK((k_tiny_residual<OffT>), 1, kBlock, r, x);
    if ((e = launch_coop(k_trim1<OffT>, c->g_coop[2], s, r, x, 0, 1, 1))) return e;
    prev_plain = false;
    if (r.flags & ISPAN_F_EXACT_STATS) PK((k_list_degrees<OffT>), G, kBlock, r, r.wl[1], x.ctl + K_WL1, C_Q2_N, C_Q2_XDEG);
    EV(5);
    PK((k_trim2<OffT>), G, kBlock, r, x, x.cand, x.ctl + K_CAND);
    EV(6);
    PK((k_trim3<OffT>), G, kBlock, r, x, x.cand, x.ctl + K_CAND);
    EV(7);
    // the first peel left its cascade counters and the consumed list count at zero
    if ((e = launch_coop(k_trim1<OffT>, c->g_coop[2], s, r, x, 1, 0, 0))) return e;
    prev_plain = false;
    EV(8);
    PK((k_wcc_init<OffT>), G, kBlock, r, x, 0);
    PK((k_wcc_hook<OffT>), G, kBlock, r, x, 0, 0);
    PK((k_wcc_compress<OffT>), G, kBlock, r, x, 0);
    if (r.nseg > 1)
        PK((k_wcc_giant_seg<OffT>), std::max<int64_t>(1, std::min<int64_t>(G, (r.nseg + kWarps - 1) / kWarps)), kBlock, r, x);
    else
        PK((k_wcc_giant<OffT>), 1, kWccRootSamples, r, x, 0);
    PK((k_wcc_hook<OffT>), G, kBlock, r, x, 0, 1);
    PK((k_wcc_flatten<OffT>), G, kBlock, r, x, 0);
    PK((k_wcc_alloc<OffT>), G, kBlock, r, x);
    PK((k_wcc_scatter<OffT>), G, kBlock, r, x, 0);
    EV(9);
    PK((k_local_scc<OffT>), c->nsm * 6, kLocalThreads, r, x);
    EV(10);
    if (c->tuning.color_compact >= 0 && r.V >= 4 * kCmpMin) {  // (smaller graphs never qualify)
        // the large WCCs' subgraph in dense ids (compact.cuh), then the
        // colouring on it; the input-graph form returns at once if it was built
        CmpBufs b;
        b.newid = c->cnt_out;
        b.old = c->small;
        b.dout = c->members;
        b.din = c->roots;
        b.fbeg = reinterpret_cast<int32_t *>(c->qe[1]);
        b.bbeg = b.fbeg + (r.V + 1);
        // adjacency: out-edges over wl[0..1], in-edges over members/roots (free
        // once the degrees they hold are scanned), 2 (maxV + 32) entries each
        b.fadj = c->wl[0];
        b.badj = c->members;
        b.bsum = reinterpret_cast<long long *>(c->aux);
        b.cap_e = 2 * (c->maxV + 32);
        b.V = r.V;
        const int nblk = (int)std::max<int64_t>(1, std::min<int64_t>(kScanBlocks, r.V / 4));
        PK((k_cmp_count<OffT>), nblk, kBlock, r, x, b);
        PK((k_cmp_tops), 1, kScanBlocks, x.ctl, b, nblk);
        PK((k_cmp_offsets<OffT>), nblk, kBlock, r, x, b);
        PK((k_cmp_fill<OffT>), G, kBlock, r, x, b);
        Run<int32_t> rc;
        Ext<int32_t> xc;
        compact_run(r, x, b, rc, xc);
        if ((e = launch_coop(k_color<int32_t>, c->g_coop[4], s, rc, xc))) return e;
        prev_plain = false;
    }
    if ((e = launch_coop(k_color<OffT>, c->g_coop[3], s, r, x))) return e;
    prev_plain = false;
    EV(11);
    PK((k_finalize<OffT>), G, kBlock, r, x);
    EV(12);
#undef EV
#undef LK
#undef PK
    return cudaSuccess;
}

template <typename OffT>
static int coop_setup(ispan_ctx *c) {
    int w = (int)sizeof(OffT);
    if (c->g_coop_w == w) return ISPAN_OK;
    // a server lane sizes its persistent grids for its share of the SMs, so
    // the lanes' persistent kernels are co-resident whatever runs at once
    const int nsm = c->nsm_coop > 0 ? c->nsm_coop : c->nsm;
    c->g_coop[0] = coop_grid(k_bfs<OffT, 0>, nsm, kBlock);
    c->g_coop[1] = coop_grid(k_bfs<OffT, 1>, nsm, kBlock);
    // fewer CTAs per SM than the occupancy limit on request (never more)
    const int want = c->tuning.bfs_ctas_per_sm;
    if (want > 0)
        for (int i = 0; i < 2; ++i) c->g_coop[i] = std::min(c->g_coop[i], want * nsm);
    // two searches at the same time: each on half of what both can keep resident
    c->g_pair = std::max(1, std::min(c->g_coop[0], c->g_coop[1]) / 2);
    c->g_coop[2] = coop_grid(k_trim1<OffT>, nsm, kBlock);
    c->g_coop[3] = coop_grid(k_color<OffT>, nsm, kBlock);
    c->g_coop[4] = coop_grid(k_color<int32_t>, nsm, kBlock);
    for (int i = 0; i < 5; ++i)
        if (c->g_coop[i] < 1) return ISPAN_ERR_CUDA;
    c->g_coop_w = w;
    return ISPAN_OK;
}

// L2 residency of the status maps: an access-policy window over the bitmap
// block on the run's stream (captured into the graph's kernel nodes), with
// the device's persisting L2 carve-out raised to cover it.  The carve-out is
// a limit of this process's context; it ends with the context.
static void l2_window(ispan_ctx *c, bool on) {
    int maxwin = 0, maxpersist = 0;
    cudaDeviceGetAttribute(&maxwin, cudaDevAttrMaxAccessPolicyWindowSize, c->device);
    cudaDeviceGetAttribute(&maxpersist, cudaDevAttrMaxPersistingL2CacheSize, c->device);
    if (maxwin <= 0 || maxpersist <= 0 || c->bits_bytes <= 0) return;
    const size_t bytes = std::min<size_t>((size_t)c->bits_bytes, (size_t)maxwin);
    size_t limit = 0;
    if (on) {
        cudaDeviceGetLimit(&limit, cudaLimitPersistingL2CacheSize);
        const size_t want = std::min<size_t>(bytes, (size_t)maxpersist);
        if (limit < want) {
            if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) != cudaSuccess) {
                cudaGetLastError();
                return;
            }
            limit = want;
        }
        c->l2_limit_set = true;
    }
    cudaStreamAttrValue v;
    memset(&v, 0, sizeof v);
    if (on) {
        v.accessPolicyWindow.base_ptr = c->bits;
        v.accessPolicyWindow.num_bytes = bytes;
        v.accessPolicyWindow.hitRatio = std::min(1.0f, (float)limit / (float)bytes);
        v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    }
    if (cudaStreamSetAttribute(c->stream, cudaStreamAttributeAccessPolicyWindow, &v) != cudaSuccess)
        cudaGetLastError();
}

template <typename OffT>
static int run_t(ispan_ctx *c, int64_t V, int64_t E, int32_t nseg, const OffT *fwb, const OffT *bwb,
                 const int32_t *fwa, const int32_t *bwa, int32_t *label_dev, const ispan_params *p,
                 ispan_stats *st) {
    int rc = coop_setup<OffT>(c);
    if (rc) return rc;
    Run<OffT> r;
    Ext<OffT> x;
    memset(&r, 0, sizeof(r));
    memset(&x, 0, sizeof(x));
    fill_run<OffT>(c, r, x, V, E, nseg, fwb, bwb, fwa, bwa, label_dev, p);
    const uint32_t flags = p ? p->flags : 0;
#ifdef ISPAN_CHECKED
    const bool validate = true;
#else
    const bool validate = (flags & ISPAN_F_VALIDATE) || c->validate_next;
#endif
    c->validate_next = false;
    if (validate) {
        CK(cudaMemsetAsync(c->err, 0, 4 * sizeof(int), c->stream));
        k_validate<OffT><<<c->g_stream, 256, 0, c->stream>>>(fwb, bwb, fwa, bwa, V, E, c->err + 1);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(c->h_err, c->err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        if (c->h_err[1]) return ISPAN_ERR_ARG;
    }
#ifdef ISPAN_CHECKED
    {
        long long caps[3] = {(long long)V, (long long)E, (long long)(c->maxE / kChunk + 4)};
        long long zero[2] = {0, 0};
        CK(cudaMemcpyToSymbolAsync(g_vcap, &caps[0], 8, 0, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyToSymbolAsync(g_ecap, &caps[1], 8, 0, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyToSymbolAsync(g_qcap, &caps[2], 8, 0, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyToSymbolAsync(g_chk, zero, 16, 0, cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
#endif
    // stage events are recorded (and captured) only when the caller asks for
    // stage times
    const bool times = (flags & ISPAN_F_STAGE_TIMES) && st && c->have_ev;
    const int ev_on = times ? 1 : 0;
    // the window pays only for maps larger than what stays in L2 anyway; on
    // small graphs its attribute calls would cost more than the run's stages
    const bool l2win = !(flags & ISPAN_F_NO_L2_WINDOW) && 6 * r.W * 4 >= kL2WindowMinBytes;
    if (l2win) l2_window(c, true);
    bool use_graph = !(flags & ISPAN_F_NO_GRAPH) && !c->graph_broken;
    if (use_graph) {
        char key[256];
        snprintf(key, sizeof key, "%d|%lld|%lld|%d|%p|%p|%p|%p|%p|%d|%d|%d|%p|%u", (int)sizeof(OffT), (long long)V,
                 (long long)E, nseg, (const void *)fwb, (const void *)bwb, (const void *)fwa, (const void *)bwa,
                 (void *)label_dev, r.alpha, r.beta, r.gamma, (void *)c->stream,
                 r.flags & (ISPAN_F_EXACT_STATS | ISPAN_F_NO_L2_WINDOW));
        // two cached graphs: with the stage-time events (requested times) and
        // without them, so a run that reads no times pays for no event nodes
        cudaGraphExec_t &gx = c->gexec[ev_on];
        char *gk = c->gkey[ev_on];
        if (!gx || strcmp(key, gk) != 0) {
            if (gx) {
                cudaGraphExecDestroy(gx);
                gx = nullptr;
            }
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
            if (e == cudaSuccess) {
                cudaError_t e2 = enqueue<OffT>(c, r, x, ev_on, true);
                e = cudaStreamEndCapture(c->stream, &g);
                if (e2 != cudaSuccess) e = e2;
            }
            if (e == cudaSuccess) e = cudaGraphInstantiate(&gx, g, 0);
            if (g) cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                cudaGetLastError();
                c->graph_broken = true;  // fall back to direct launches from now on
                gx = nullptr;
                use_graph = false;
            } else {
                snprintf(gk, sizeof c->gkey[0], "%s", key);
            }
        }
    }
    if (use_graph) {
        CK(cudaGraphLaunch(c->gexec[ev_on], c->stream));
    } else {
        CK(enqueue<OffT>(c, r, x, ev_on, false));
    }
    CK(cudaMemcpyAsync(c->h_counters, c->ctlblk, kNumCounters * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->h_err, c->err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (l2win) l2_window(c, false);  // the caller's stream gets its attribute back
#ifdef ISPAN_CHECKED
    {
        long long chk[2] = {0, 0};
        CK(cudaMemcpyFromSymbol(chk, g_chk, 16));
        if (chk[0]) {
            fprintf(stderr, "ispan_b200 (checked build): range check failed at site %lld, index %lld\n", chk[0],
                    chk[1]);
            return ISPAN_ERR_INTERNAL;
        }
    }
#endif
    if (c->h_err[0]) return c->h_err[0] < 0 ? c->h_err[0] : ISPAN_ERR_INTERNAL;
    if (st) {
        const unsigned long long *k = c->h_counters;
        memset(st->stage_ms, 0, sizeof(st->stage_ms));
        st->giant_size = (int64_t)k[C_GIANT];
        st->n_trim1 = (int64_t)k[C_TRIM1];
        st->n_trim2 = (int64_t)k[C_TRIM2];
        st->n_trim3 = (int64_t)k[C_TRIM3];
        st->n_mice_vertices = (int64_t)k[C_MICE_V];
        st->n_mice_scc = (int64_t)k[C_MICE_SCC];
        st->n_wcc = (int64_t)k[C_WCC];
        st->fw_size = (int64_t)k[C_FW_SIZE];
        st->fw_levels = (int64_t)k[C_FW_LEVELS];
        st->bw_levels = (int64_t)k[C_BW_LEVELS];
        st->color_rounds = (int64_t)k[C_COLOR_ROUNDS];
        st->local_wcc = (int64_t)k[C_LOCAL_WCC];
        st->trim_rounds = (int64_t)k[C_TRIM_ROUNDS];
        st->residual = (int64_t)(k[C_ACTIVE0] - k[C_GIANT]);
        st->fw_edges = (int64_t)k[C_FW_XDEG];
        st->bw_edges = (int64_t)k[C_BW_XDEG];
        st->resid_edges = (int64_t)k[C_Q1_XDEG];
        st->peeled_residual = (int64_t)k[C_Q2_N];
        st->peeled_residual_edges = (int64_t)k[C_Q2_XDEG];
        st->scc_count = (int64_t)(k[C_TRIM1] + k[C_TRIM2] / 2 + k[C_TRIM3] / 3 + k[C_MICE_SCC] + k[C_GIANTS]);
        if (times) {
            float ms[kNumEv];
            for (int i = 1; i < kNumEv; ++i) cudaEventElapsedTime(&ms[i], c->ev[i - 1], c->ev[i]);
            // reference slots: 0 trim, 1 elephant, 2 mice, 3 total, 4 trim size_1,
            // 5 trim size_2, 6 pivot, 7 fw, 8 bw, 9 wcc, 10 mice fw-bw, 13 trim size_3;
            // finer slots of this engine: 11 large-WCC colouring (part of 10),
            // 12 second peel, 14 residual worklist after the pivot SCCs, 15 first
            // peel (12, 14 and 15 are parts of 4)
            st->stage_ms[6] = ms[1];
            st->stage_ms[7] = ms[2];
            st->stage_ms[8] = ms[3];
            st->stage_ms[14] = ms[4];
            st->stage_ms[15] = ms[5];
            st->stage_ms[12] = ms[8];
            st->stage_ms[4] = ms[1] + ms[4] + ms[5] + ms[8];
            st->stage_ms[5] = ms[6];
            st->stage_ms[13] = ms[7];
            st->stage_ms[9] = ms[9];
            st->stage_ms[11] = ms[11];
            st->stage_ms[10] = ms[10] + ms[11];
            st->stage_ms[0] = st->stage_ms[4] + st->stage_ms[5] + st->stage_ms[13];
            st->stage_ms[1] = ms[2] + ms[3];
            st->stage_ms[2] = st->stage_ms[9] + st->stage_ms[10];
            float tot = 0;
            cudaEventElapsedTime(&tot, c->ev[0], c->ev[kNumEv - 1]);
            st->stage_ms[3] = tot;
        }
        st->hist_n = 0;
        if (st->hist_size && st->hist_count && st->hist_cap > 0) {
            std::vector<int64_t> h(kHistCap + kBigCap);
            CK(cudaMemcpy(h.data(), c->hist, h.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
            std::vector<std::pair<int64_t, int64_t>> pairs;
            for (int i = 1; i < kHistCap; ++i)
                if (h[i]) pairs.push_back({i, h[i]});
            int64_t nbig = std::min<int64_t>((int64_t)k[C_BIG], kBigCap);
            std::vector<int64_t> big(h.begin() + kHistCap, h.begin() + kHistCap + nbig);
            std::sort(big.begin(), big.end());
            for (size_t i = 0; i < big.size();) {
                size_t j = i;
                while (j < big.size() && big[j] == big[i]) ++j;
                pairs.push_back({big[i], (int64_t)(j - i)});
                i = j;
            }
            st->hist_n = (int64_t)pairs.size();
            for (int64_t i = 0; i < st->hist_n && i < st->hist_cap; ++i) {
                st->hist_size[i] = pairs[i].first;
                st->hist_count[i] = pairs[i].second;
            }
        }
    }
    c->last_V = V;
    c->last_label = label_dev;
    c->last_nseg = nseg;
    return ISPAN_OK;
}

// a CSR that gives the forward direction only (bw_beg and bw_adj both NULL):
// the run builds the reverse on the device
static bool fw_only(const ispan_csr *g) { return g && !g->bw_beg && !g->bw_adj; }

static int check_csr(const ispan_csr *g, bool allow_fw_only = false) {
    if (!g || g->V < 0 || g->E < 0) return ISPAN_ERR_ARG;
    if (g->offset_bytes != 4 && g->offset_bytes != 8) return ISPAN_ERR_ARG;
    if (g->offset_bytes == 4 && g->E > INT32_MAX) return ISPAN_ERR_ARG;
    if (g->V >= INT32_MAX) return ISPAN_ERR_ARG;
    const bool rev = !(allow_fw_only && fw_only(g));
    if (g->V > 0 && (!g->fw_beg || (rev && !g->bw_beg))) return ISPAN_ERR_ARG;
    if (g->E > 0 && (!g->fw_adj || (rev && !g->bw_adj))) return ISPAN_ERR_ARG;
    return ISPAN_OK;
}

// chunks of the forward adjacency's copy: at least 2^22 ids each (a small
// graph's copy is one chunk: the launches would cost more than the overlap
// gains), at most kUpChunks, boundaries on multiples of four ids (the count
// reads int4)
static int up_chunks(int64_t E, int64_t *step) {
    const int nch = (int)std::max<int64_t>(1, std::min<int64_t>(kUpChunks, E >> 22));
    *step = ((E + nch - 1) / nch + 3) / 4 * 4;
    return nch;
}

// scratch of the sorted reverse lists for V vertices and E edges (2 E ids,
// two chunks' alternates, kUpChunks + 1 arrays of V counts, the sort's and
// the scan's storage; kept for later runs); false if it does not fit
static bool ensure_rev_sort(ispan_ctx *c, int64_t V, int64_t E) {
    if (!c->rv_failed && c->rv_E >= E && c->rv_V >= V) return true;
    if (c->rv_failed && E >= c->rv_E && V >= c->rv_V) return false;
    for (void *p : c->rv_owned) cudaFree(p);
    c->rv_owned.clear();
    c->rv_E = c->rv_V = -1;
    int64_t step = 0;
    up_chunks(E, &step);
    size_t tb = 0, ts = 0;
    cub::DoubleBuffer<int32_t> k(nullptr, nullptr), v(nullptr, nullptr);
    bool ok = cub::DeviceRadixSort::SortPairs(nullptr, tb, k, v, (int)step, 0, 32, c->stream) == cudaSuccess &&
              cub::DeviceScan::ExclusiveSum(nullptr, ts, (int32_t *)nullptr, (int32_t *)nullptr, (int)V,
                                            c->stream) == cudaSuccess;
    tb = std::max(tb, ts);
    ok = ok && dalloc(&c->rv_k0, (size_t)E, c->rv_owned) == 0 && dalloc(&c->rv_v, (size_t)E, c->rv_owned) == 0 &&
         dalloc(&c->rv_k1, (size_t)step, c->rv_owned) == 0 && dalloc(&c->rv_v1, (size_t)step, c->rv_owned) == 0 &&
         dalloc(&c->rv_snap, (size_t)kUpChunks * V, c->rv_owned) == 0 &&
         dalloc(&c->rv_run, (size_t)V, c->rv_owned) == 0 && dalloc((char **)&c->rv_tmp, tb, c->rv_owned) == 0;
    if (!ok) {
        for (void *p : c->rv_owned) cudaFree(p);
        c->rv_owned.clear();
        cudaGetLastError();  // a failed allocation is not an error of the run
        c->rv_failed = true;
        c->rv_E = E;  // this size (and larger) takes the atomic placement
        c->rv_V = V;
        return false;
    }
    c->rv_tmp_bytes = tb;
    c->rv_E = E;
    c->rv_V = V;
    c->rv_failed = false;
    return true;
}

// the verdict of the reverse build's checks on the forward CSR
static int rev_checked(ispan_ctx *c) {
    CK(cudaMemcpyAsync(c->h_err + 2, c->err + 2, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return c->h_err[2] ? ISPAN_ERR_ARG : ISPAN_OK;
}

// The reverse CSR (X = reverse offsets, ba = reverse adjacency) of the
// forward CSR (fb, fa) on the device.  With `host` set, fb and fa are host
// arrays: the offsets and then the adjacency, in kUpChunks chunks, are
// copied into dfb/dfa on c->stream, and each chunk's in-degrees are counted
// on c->stream2 as soon as it has landed, so counting overlaps the copy.
template <typename OffT>
static int build_reverse(ispan_ctx *c, int64_t V, int64_t E, const OffT *fb, const int32_t *fa, OffT *dfb,
                         int32_t *dfa, bool host, OffT *X, int32_t *ba, bool atomic) {
    cudaStream_t s = c->stream, s2 = c->stream2;
    int pc = 0, pf = 0;  // resident CTAs per SM of each kernel: a full grid
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pc, k_rev_count<OffT>, kBlock, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pf, k_rev_fill<OffT>, kBlock, 0);
    const int gc = std::max(1, pc) * c->nsm, gf = std::max(1, pf) * c->nsm;
    for (int k = 0; k < kUpChunks; ++k)
        if (!c->ev_up[k] && cudaEventCreateWithFlags(&c->ev_up[k], cudaEventDisableTiming) != cudaSuccess)
            return ISPAN_ERR_CUDA;
    size_t need = 0;
    CK(cub::DeviceScan::InclusiveSum(nullptr, need, X, X, (int)V, s));
    if (need > c->scan_tmp_bytes) {
        if (c->scan_tmp) cudaFree(c->scan_tmp);
        c->scan_tmp = nullptr;
        c->scan_tmp_bytes = 0;
        if (cudaMalloc(&c->scan_tmp, need) != cudaSuccess) return ISPAN_ERR_NOMEM;
        c->scan_tmp_bytes = need;
    }
    int *bad = c->err + 2;  // a malformed forward CSR, seen by the passes below
    CK(cudaMemsetAsync(bad, 0, sizeof(int), s));
    int64_t step = 0;
    const int nch = up_chunks(E, &step);
    // the lists by a sort of each chunk where the scratch fits (chunks below
    // 2^31 edges); the counts then go one slot up (X[w + 1]), so that their
    // inclusive scan is the start offsets
    const bool sorted = !atomic && E > 0 && step < INT32_MAX && ensure_rev_sort(c, V, E);
    OffT *cnt = sorted ? X + 1 : X;
    int bits = 1;  // key bits of the sort: ids below V
    while (bits < 31 && (1ll << bits) < V) ++bits;
    CK(cudaMemsetAsync(X, 0, (size_t)(V + 1) * sizeof(OffT), s));
    if (host) CK(cudaMemcpyAsync(dfb, fb, (size_t)(V + 1) * sizeof(OffT), cudaMemcpyHostToDevice, s));
    if (sorted) {
        // the sort's values (each edge's source) need the offsets only: they
        // are written while the adjacency is still being copied
        CK(cudaEventRecord(c->ev_fork, s));
        CK(cudaStreamWaitEvent(s2, c->ev_fork, 0));
        k_rev_sources<OffT><<<gf, kBlock, 0, s2>>>(dfb, V, E, c->rv_v, bad);
        CK(cudaGetLastError());
    }
    // each chunk, as soon as it has landed: its in-degree counts and, for the
    // sort, a snapshot of the running counts, its keys (a copy of the ids:
    // the forward lists must survive) and its own stable sort
    for (int k = 0; k < nch; ++k) {
        const int64_t e0 = std::min<int64_t>(E, k * step), e1 = std::min<int64_t>(E, e0 + step);
        if (host && e1 > e0)
            CK(cudaMemcpyAsync(dfa + e0, fa + e0, (size_t)(e1 - e0) * 4, cudaMemcpyHostToDevice, s));
        CK(cudaEventRecord(c->ev_up[k], s));
        CK(cudaStreamWaitEvent(s2, c->ev_up[k], 0));
        if (e1 > e0) {
            k_rev_count<OffT><<<gc, kBlock, 0, s2>>>(dfa, e0, e1, V, cnt, bad);
            CK(cudaGetLastError());
        }
        if (!sorted) continue;
        k_rev_snap<OffT><<<gf, kBlock, 0, s2>>>(cnt, V, c->rv_snap + (size_t)k * V);
        CK(cudaGetLastError());
        if (e1 > e0) {
            const int n = (int)(e1 - e0);
            CK(cudaMemcpyAsync(c->rv_k0 + e0, dfa + e0, (size_t)n * 4, cudaMemcpyDeviceToDevice, s2));
            cub::DoubleBuffer<int32_t> keys(c->rv_k0 + e0, c->rv_k1), vals(c->rv_v + e0, c->rv_v1);
            size_t tb = c->rv_tmp_bytes;
            CK(cub::DeviceRadixSort::SortPairs(c->rv_tmp, tb, keys, vals, n, 0, bits, s2));
            if (keys.Current() != c->rv_k0 + e0)
                CK(cudaMemcpyAsync(c->rv_k0 + e0, keys.Current(), (size_t)n * 4, cudaMemcpyDeviceToDevice, s2));
            if (vals.Current() != c->rv_v + e0)
                CK(cudaMemcpyAsync(c->rv_v + e0, vals.Current(), (size_t)n * 4, cudaMemcpyDeviceToDevice, s2));
        }
    }
    CK(cudaEventRecord(c->ev_join, s2));
    CK(cudaStreamWaitEvent(s, c->ev_join, 0));
    if (V > 0) CK(cub::DeviceScan::InclusiveSum(c->scan_tmp, need, cnt, cnt, (int)V, s));
    if (!sorted) {
        k_rev_fill<OffT><<<gf, kBlock, 0, s>>>(dfb, dfa, V, E, X, ba, bad);
        CK(cudaGetLastError());
        return rev_checked(c);
    }
    // each chunk's sorted runs into place: run starts inside the chunk (the
    // exclusive scan of its own counts), then the pairs
    for (int k = 0; k < nch; ++k) {
        const int64_t e0 = std::min<int64_t>(E, k * step), e1 = std::min<int64_t>(E, e0 + step);
        if (e1 <= e0) continue;
        const int32_t *before = k ? c->rv_snap + (size_t)(k - 1) * V : nullptr;
        k_rev_diff<<<gf, kBlock, 0, s>>>(c->rv_snap + (size_t)k * V, before, V, c->rv_run);
        CK(cudaGetLastError());
        size_t tb = c->rv_tmp_bytes;
        CK(cub::DeviceScan::ExclusiveSum(c->rv_tmp, tb, c->rv_run, c->rv_run, (int)V, s));
        k_rev_runs<OffT><<<gf, kBlock, 0, s>>>(c->rv_k0 + e0, c->rv_v + e0, e1 - e0, X, before, c->rv_run, V, ba);
        CK(cudaGetLastError());
    }
    return rev_checked(c);
}

// device buffers of an uploaded graph (and of a reverse CSR built here),
// grown on demand
static int ensure_up(ispan_ctx *c, int64_t V, int64_t E) {
    if (c->up_V >= V && c->up_E >= E && c->up_fw_beg != nullptr) return ISPAN_OK;
    for (void *p : c->csr_owned) cudaFree(p);
    c->csr_owned.clear();
    int rc = 0;
    char *a = nullptr, *b = nullptr;
    rc |= dalloc(&a, (size_t)(V + 1) * 8, c->csr_owned);
    rc |= dalloc(&b, (size_t)(V + 1) * 8, c->csr_owned);
    rc |= dalloc(&c->up_fw_adj, (size_t)E, c->csr_owned);
    rc |= dalloc(&c->up_bw_adj, (size_t)E, c->csr_owned);
    if (rc) {
        c->up_V = c->up_E = -1;
        c->up_fw_beg = nullptr;
        return ISPAN_ERR_NOMEM;
    }
    c->up_fw_beg = a;
    c->up_bw_beg = b;
    c->up_V = V;
    c->up_E = E;
    return ISPAN_OK;
}

// Host input: the copies' sizes come from V and E alone; the offsets and ids
// are checked on the device before any stage reads them.  A forward-only
// graph is copied in one direction and its reverse built on the device.
static int upload(ispan_ctx *c, const ispan_csr *g, bool atomic) {
    int rc = ensure_up(c, g->V, g->E);
    if (rc) return rc;
    if (fw_only(g)) {
        if (g->offset_bytes == 4)
            return build_reverse<int32_t>(c, g->V, g->E, (const int32_t *)g->fw_beg, g->fw_adj,
                                          (int32_t *)c->up_fw_beg, c->up_fw_adj, true, (int32_t *)c->up_bw_beg,
                                          c->up_bw_adj, atomic);
        return build_reverse<int64_t>(c, g->V, g->E, (const int64_t *)g->fw_beg, g->fw_adj, (int64_t *)c->up_fw_beg,
                                      c->up_fw_adj, true, (int64_t *)c->up_bw_beg, c->up_bw_adj, atomic);
    }
    size_t ob = (size_t)g->offset_bytes;
    CK(cudaMemcpyAsync(c->up_fw_beg, g->fw_beg, (size_t)(g->V + 1) * ob, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->up_bw_beg, g->bw_beg, (size_t)(g->V + 1) * ob, cudaMemcpyHostToDevice, c->stream));
    if (g->E) {
        CK(cudaMemcpyAsync(c->up_fw_adj, g->fw_adj, (size_t)g->E * 4, cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->up_bw_adj, g->bw_adj, (size_t)g->E * 4, cudaMemcpyHostToDevice, c->stream));
    }
    return ISPAN_OK;
}

// the body of a run; the caller holds c->mu and has made c->device current
static int run_locked(ispan_ctx *c, const ispan_csr *g, int32_t nseg, const int64_t *vbase_host,
                      const ispan_params *p, int32_t *labels_out, ispan_stats *st) {
    int rc = check_csr(g, true);
    if (rc) return rc;
    if (g->V > c->maxV || g->E > c->maxE) return ISPAN_ERR_CAPACITY;
    if (nseg < 1) return ISPAN_ERR_ARG;
    if ((rc = ctx_segments(c, nseg))) return rc;
    std::vector<int64_t> vb;
    if (vbase_host) {
        vb.assign(vbase_host, vbase_host + nseg + 1);
        if (vb[0] != 0 || vb[nseg] != g->V) return ISPAN_ERR_ARG;
        for (int i = 0; i < nseg; ++i)
            if (vb[i + 1] < vb[i]) return ISPAN_ERR_ARG;
    } else {
        vb = {0, g->V};
    }
    if (vb != c->vbase_host) {  // upload only when the segmentation changed
        CK(cudaMemcpyAsync(c->vbase, vb.data(), vb.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->stream));
        CK(cudaStreamSynchronize(c->stream));  // vb is a host temporary
        c->vbase_host = vb;
    }
    const void *fwb = g->fw_beg, *bwb = g->bw_beg;
    const int32_t *fwa = g->fw_adj, *bwa = g->bw_adj;
    const bool atomic = p && (p->flags & ISPAN_F_REVERSE_ATOMIC);
    if (!g->on_device) {
        // the copies' sizes come from V and E alone; the offsets (monotone,
        // from 0 to E) and the ids of host input are checked on the device,
        // before any stage reads them (a serial host scan of the offsets
        // cost more than the upload itself on large graphs)
        if ((rc = upload(c, g, atomic))) return rc;
        // a forward-only graph was checked while its reverse was built
        c->validate_next = !fw_only(g) || g->V == 0;
        fwb = c->up_fw_beg;
        bwb = c->up_bw_beg;
        fwa = c->up_fw_adj;
        bwa = c->up_bw_adj;
    } else if (fw_only(g)) {
        // device input in one direction: the reverse goes to the upload
        // buffers, and the forward CSR is checked while it is built
        if ((rc = ensure_up(c, g->V, g->E))) return rc;
        if (g->offset_bytes == 4)
            rc = build_reverse<int32_t>(c, g->V, g->E, (const int32_t *)fwb, fwa, (int32_t *)fwb,
                                        const_cast<int32_t *>(fwa), false, (int32_t *)c->up_bw_beg, c->up_bw_adj,
                                        atomic);
        else
            rc = build_reverse<int64_t>(c, g->V, g->E, (const int64_t *)fwb, fwa, (int64_t *)fwb,
                                        const_cast<int32_t *>(fwa), false, (int64_t *)c->up_bw_beg, c->up_bw_adj,
                                        atomic);
        if (rc) return rc;
        c->validate_next = g->V == 0;  // checked while the reverse was built
        bwb = c->up_bw_beg;
        bwa = c->up_bw_adj;
    }
    const bool dev_labels = p && (p->flags & ISPAN_F_LABELS_ON_DEVICE);
    int32_t *label = dev_labels ? labels_out : c->label;
    if (!label && g->V) return ISPAN_ERR_ARG;
    if (g->offset_bytes == 4)
        rc = run_t<int32_t>(c, g->V, g->E, nseg, (const int32_t *)fwb, (const int32_t *)bwb, fwa, bwa, label, p, st);
    else
        rc = run_t<int64_t>(c, g->V, g->E, nseg, (const int64_t *)fwb, (const int64_t *)bwb, fwa, bwa, label, p, st);
    if (rc) return rc;
    if (!dev_labels && labels_out && g->V) {
        CK(cudaMemcpyAsync(labels_out, c->label, (size_t)g->V * 4, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return ISPAN_OK;
}

static int run_common(ispan_ctx *c, const ispan_csr *g, int32_t nseg, const int64_t *vbase_host,
                      const ispan_params *p, int32_t *labels_out, ispan_stats *st) {
    if (!c) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return ISPAN_ERR_CUDA;
    return run_locked(c, g, nseg, vbase_host, p, labels_out, st);
}

// union buffers for ispan_scc_run_graphs: the CSR at the context's capacity
// on first use, the per-graph tables grown to n (device tables from the
// lane's region when the context is bound to one; pinned host mirrors always
// from cudaMallocHost)
static int pk_reserve(ispan_ctx *c, int64_t n) {
    if (!c->pk_fwb) {
        int rc = 0;
        rc |= dalloc(&c->pk_fwb, c->maxV + 1, c->pk_owned, c->rg);
        rc |= dalloc(&c->pk_bwb, c->maxV + 1, c->pk_owned, c->rg);
        rc |= dalloc(&c->pk_fwa, c->maxE, c->pk_owned, c->rg);
        rc |= dalloc(&c->pk_bwa, c->maxE, c->pk_owned, c->rg);
        if (rc) {
            for (void *q : c->pk_owned) cudaFree(q);
            c->pk_owned.clear();
            c->pk_fwb = c->pk_bwb = nullptr;
            c->pk_fwa = c->pk_bwa = nullptr;
            return ISPAN_ERR_NOMEM;
        }
    }
    if (n > c->h_cap) {
        const int64_t m = std::max<int64_t>({n, 2 * c->h_cap, 64});
        if (c->h_desc) cudaFreeHost(c->h_desc);
        if (c->h_vbeb) cudaFreeHost(c->h_vbeb);
        c->h_desc = nullptr;
        c->h_vbeb = nullptr;
        c->h_cap = 0;
        if (cudaMallocHost(&c->h_desc, m * sizeof(PackDesc)) != cudaSuccess ||
            cudaMallocHost(&c->h_vbeb, 2 * (m + 1) * sizeof(int64_t)) != cudaSuccess) {
            cudaGetLastError();
            return ISPAN_ERR_NOMEM;
        }
        c->h_cap = m;
    }
    if (n <= c->pk_n) return ISPAN_OK;
    if (c->rg && c->pk_n > 0) return ISPAN_ERR_CAPACITY;  // a lane's tables were carved for its batch
    const int64_t m = c->rg ? std::max<int64_t>(n, 1) : std::max<int64_t>({n, 2 * c->pk_n, 64});
    if (!c->rg) {
        for (void *q : c->pkt_owned) cudaFree(q);
        c->pkt_owned.clear();
    }
    c->pk_n = 0;
    int rc = 0;
    rc |= dalloc(&c->pk_desc, m, c->pkt_owned, c->rg);
    rc |= dalloc(&c->pk_vb, 2 * (m + 1), c->pkt_owned, c->rg);
    rc |= dalloc(&c->pk_stage, 2 * ((c->stage_V >= 0 ? c->stage_V : c->maxV) + m), c->pkt_owned, c->rg);
    if (rc) return ISPAN_ERR_NOMEM;
    c->pk_eb = c->pk_vb + (m + 1);
    c->pk_n = m;
    return ISPAN_OK;
}

// phase 1 of ispan_scc_run_graphs: the union of gs in the context's union
// buffers, checked; the segmentation is kept for phase 2
static int pack_graphs(ispan_ctx *c, const ispan_csr *gs, int32_t n) {
    c->pk_ready = false;
    int64_t Vt = 0, Et = 0;
    for (int32_t i = 0; i < n; ++i) {
        int rc = check_csr(&gs[i]);
        if (rc) return rc;
        Vt += gs[i].V;
        Et += gs[i].E;
    }
    if (Vt > c->maxV || Et > c->maxE) return ISPAN_ERR_CAPACITY;
    // host graphs' offsets are checked on the device by k_pack_offsets, like
    // the device graphs' (the adjacency is packed by edge slot, so no access
    // depends on an offset before the check)
    int rc = pk_reserve(c, n);
    if (rc) return rc;
    cudaStream_t s = c->stream;
    // the previous batch may still read the pinned tables
    CK(cudaStreamSynchronize(s));
    PackDesc *hd = c->h_desc;
    int64_t *hvb = c->h_vbeb, *heb = c->h_vbeb + (n + 1);
    int64_t vb = 0, eb = 0, so = 0;
    for (int32_t i = 0; i < n; ++i) {
        const ispan_csr &g = gs[i];
        PackDesc d;
        memset(&d, 0, sizeof d);
        d.V = g.V;
        d.E = g.E;
        d.vbase = vb;
        d.ebase = eb;
        d.ob = g.offset_bytes;
        hvb[i] = vb;
        heb[i] = eb;
        if (g.on_device) {
            d.fw_beg = g.fw_beg;
            d.bw_beg = g.bw_beg;
            d.fw_adj = g.fw_adj;
            d.bw_adj = g.bw_adj;
        } else {
            // offsets staged as they are; adjacency straight into its union
            // slice, where k_pack_adj adds the vertex base in place
            const size_t ob = (size_t)g.offset_bytes;
            char *st0 = reinterpret_cast<char *>(c->pk_stage + so);
            char *st1 = reinterpret_cast<char *>(c->pk_stage + so + (g.V + 1));
            if (g.V > 0 || g.E > 0) {
                CK(cudaMemcpyAsync(st0, g.fw_beg, (size_t)(g.V + 1) * ob, cudaMemcpyHostToDevice, s));
                CK(cudaMemcpyAsync(st1, g.bw_beg, (size_t)(g.V + 1) * ob, cudaMemcpyHostToDevice, s));
            }
            so += 2 * (g.V + 1);
            if (g.E) {
                CK(cudaMemcpyAsync(c->pk_fwa + eb, g.fw_adj, (size_t)g.E * 4, cudaMemcpyHostToDevice, s));
                CK(cudaMemcpyAsync(c->pk_bwa + eb, g.bw_adj, (size_t)g.E * 4, cudaMemcpyHostToDevice, s));
            }
            d.fw_beg = st0;
            d.bw_beg = st1;
            d.fw_adj = c->pk_fwa + eb;
            d.bw_adj = c->pk_bwa + eb;
        }
        hd[i] = d;
        vb += g.V;
        eb += g.E;
    }
    hvb[n] = Vt;
    heb[n] = Et;
    CK(cudaMemcpyAsync(c->pk_desc, hd, n * sizeof(PackDesc), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(c->pk_vb, hvb, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(c->pk_eb, heb, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(c->err, 0, 4 * sizeof(int), s));
    const int64_t tiles_v = Vt / kPackTile + 1, tiles_e = Et / kPackTile + 1;
    const int gv = (int)std::min<int64_t>(tiles_v, 8 * c->nsm), ge = (int)std::min<int64_t>(tiles_e, 8 * c->nsm);
    k_pack_offsets<<<gv, kPackThreads, 0, s>>>(c->pk_desc, n, c->pk_vb, Vt, Et, c->pk_fwb, c->pk_bwb, c->err + 1);
    CK(cudaGetLastError());
    if (Et > 0) {
        k_pack_adj<<<ge, kPackThreads, 0, s>>>(c->pk_desc, n, c->pk_eb, Et, c->pk_fwa, c->pk_bwa, c->err + 1);
        CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(c->h_err, c->err, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (c->h_err[1]) return ISPAN_ERR_ARG;
    c->pk_vbase.assign(hvb, hvb + n + 1);
    c->pk_cur_n = n;
    c->pk_Et = Et;
    c->pk_ready = true;
    return ISPAN_OK;
}

// phase 2: the pipeline over the packed union, then every graph's labels
static int run_packed(ispan_ctx *c, const ispan_csr *gs, int32_t n, int32_t *const *labels_out,
                      const ispan_params *p, ispan_stats *st) {
    if (!c->pk_ready || c->pk_cur_n != n) return ISPAN_ERR_ARG;
    for (int32_t i = 0; i < n; ++i)
        if (gs[i].V != c->pk_vbase[i + 1] - c->pk_vbase[i] || (gs[i].V > 0 && !labels_out[i])) return ISPAN_ERR_ARG;
    c->pk_ready = false;  // the union is consumed (labels overwrite the scratch)
    cudaStream_t s = c->stream;
    const std::vector<int64_t> vbase = c->pk_vbase;
    const int64_t Vt = vbase[n], Et = c->pk_Et;
    const int gv = (int)std::min<int64_t>(Vt / kPackTile + 1, 8 * c->nsm);
    int rc = 0;
    ispan_csr u;
    memset(&u, 0, sizeof u);
    u.V = Vt;
    u.E = Et;
    u.fw_beg = c->pk_fwb;
    u.bw_beg = c->pk_bwb;
    u.fw_adj = c->pk_fwa;
    u.bw_adj = c->pk_bwa;
    u.offset_bytes = 8;
    u.on_device = 1;
    ispan_params q = p ? *p : ispan_params{30, 200, 10, 0.1, 0};
    q.flags = (q.flags | ISPAN_F_LABELS_ON_DEVICE) & ~(uint32_t)ISPAN_F_VALIDATE;  // packed = checked
    if ((rc = run_locked(c, &u, n, vbase.data(), &q, c->label, st))) return rc;
    if (Vt > 0) {
        k_unpack_labels<<<gv, kPackThreads, 0, s>>>(c->label, n, c->pk_vb, Vt);
        CK(cudaGetLastError());
    }
    for (int32_t i = 0; i < n; ++i)
        if (gs[i].V > 0)
            CK(cudaMemcpyAsync(labels_out[i], c->label + vbase[i], (size_t)gs[i].V * 4, cudaMemcpyDefault, s));
    CK(cudaStreamSynchronize(s));
    return ISPAN_OK;
}

static int run_graphs(ispan_ctx *c, const ispan_csr *gs, int32_t n, int32_t *const *labels_out,
                      const ispan_params *p, ispan_stats *st) {
    for (int32_t i = 0; i < n; ++i)
        if (gs[i].V > 0 && !labels_out[i]) return ISPAN_ERR_ARG;
    int rc = pack_graphs(c, gs, n);
    return rc ? rc : run_packed(c, gs, n, labels_out, p, st);
}

// ---------------------------------------------------------------------------
// Server lanes (server.cu): a context whose scratch and union buffers are
// carved, per batch, out of a region of the server's device-memory budget.

// Carve every scratch array for a batch of n graphs with V vertices and E
// edges in total; with a null base the region only measures.
static int ctx_carve(ispan_ctx *c, int64_t V, int64_t E, int64_t n, int64_t V_host) {
    c->maxV = V;
    c->maxE = E;
    c->stage_V = V_host;  // only host graphs' offsets are staged
    c->maxSeg = 0;
    c->pk_fwb = c->pk_bwb = nullptr;
    c->pk_fwa = c->pk_bwa = nullptr;
    c->pk_n = 0;
    c->pk_ready = false;
    int rc = ctx_alloc(c);
    if (!rc) rc = ctx_segments(c, std::max<int64_t>(n, 1));
    if (!rc) rc = pk_reserve(c, std::max<int64_t>(n, 1));
    return rc;
}

size_t lane_region_bytes(int64_t V, int64_t E, int64_t n, int64_t V_host) {
    ispan_ctx m;
    Region r;  // null base: measure only
    m.rg = &r;
    m.h_cap = INT64_MAX;  // no pinned mirrors for a measurement
    ctx_carve(&m, V, E, n, V_host);
    m.rg = nullptr;
    return r.used + 256;
}

int lane_bind(ispan_ctx *c, void *base, size_t bytes, int64_t V, int64_t E, int64_t n, int64_t V_host) {
    std::lock_guard<std::mutex> lock(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return ISPAN_ERR_CUDA;
    Region &r = c->lane_region;
    r.base = (char *)base;
    r.cap = bytes;
    r.used = (size_t)((256 - ((uintptr_t)base & 255)) & 255);
    c->rg = &r;
    drop_graphs(c);  // the captured graph holds the previous batch's pointers
    c->vbase_host.clear();
    c->g_coop_w = 0;
    const int rc = ctx_carve(c, V, E, n, V_host);
    if (rc) {
        c->rg = nullptr;
        c->maxV = c->maxE = 0;
    }
    return rc;
}

void lane_unbind(ispan_ctx *c) {
    std::lock_guard<std::mutex> lock(c->mu);
    c->rg = nullptr;
    c->stage_V = -1;
    c->maxV = c->maxE = c->maxSeg = 0;  // nothing runs on a lane between batches
    c->pk_fwb = c->pk_bwb = nullptr;
    c->pk_fwa = c->pk_bwa = nullptr;
    c->pk_n = 0;
    c->pk_ready = false;
    c->last_V = 0;
}

int lane_set_sm_share(ispan_ctx *c, int nsm) {
    std::lock_guard<std::mutex> lock(c->mu);
    c->nsm_coop = std::max(1, std::min(nsm, c->nsm));
    c->g_coop_w = 0;
    return ISPAN_OK;
}

// pinned host mirrors for batches of up to n graphs, allocated once per lane
// (freeing pinned memory later would synchronise the device)
int lane_reserve_host(ispan_ctx *c, int64_t n) {
    std::lock_guard<std::mutex> lock(c->mu);
    if (n <= c->h_cap) return ISPAN_OK;
    if (c->h_desc) cudaFreeHost(c->h_desc);
    if (c->h_vbeb) cudaFreeHost(c->h_vbeb);
    c->h_desc = nullptr;
    c->h_vbeb = nullptr;
    c->h_cap = 0;
    if (cudaMallocHost(&c->h_desc, n * sizeof(PackDesc)) != cudaSuccess ||
        cudaMallocHost(&c->h_vbeb, 2 * (n + 1) * sizeof(int64_t)) != cudaSuccess) {
        cudaGetLastError();
        return ISPAN_ERR_NOMEM;
    }
    c->h_cap = n;
    return ISPAN_OK;
}

extern "C" {

int ispan_ctx_create(int device, int64_t max_V, int64_t max_E, ispan_ctx **out) {
    if (!out || max_V < 0 || max_E < 0 || max_V >= INT32_MAX) return ISPAN_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return ISPAN_ERR_NODEV;
    }
    if (device < 0 || device >= ndev) return ISPAN_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return ISPAN_ERR_CUDA;
    ispan_ctx *c = new ispan_ctx();
    c->device = device;
    c->maxV = max_V;
    c->maxE = max_E;
    cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device);
    int rc = ctx_alloc(c);
    if (!rc) rc = ctx_segments(c, 1);
    if (!rc && cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) rc = ISPAN_ERR_CUDA;
    c->own_stream = true;
    if (!rc && cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking) != cudaSuccess) rc = ISPAN_ERR_CUDA;
    if (!rc && (cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess))
        rc = ISPAN_ERR_CUDA;
    if (!rc && cudaMallocHost(&c->h_counters, kNumCounters * sizeof(unsigned long long)) != cudaSuccess)
        rc = ISPAN_ERR_NOMEM;
    if (!rc && cudaMallocHost(&c->h_err, 4 * sizeof(int)) != cudaSuccess) rc = ISPAN_ERR_NOMEM;
    if (!rc) {
        for (int i = 0; i < kNumEv; ++i)
            if (cudaEventCreate(&c->ev[i]) != cudaSuccess) rc = ISPAN_ERR_CUDA;
        c->have_ev = rc == 0;
    }
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trim1_first<int64_t>, kBlock, 0);
    c->g_stream = std::max(1, per) * c->nsm;
    if (rc) {
        cudaGetLastError();
        ispan_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return ISPAN_OK;
}

int ispan_ctx_destroy(ispan_ctx *c) {
    if (!c) return ISPAN_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    for (void *p : c->owned) cudaFree(p);
    for (void *p : c->seg_owned) cudaFree(p);
    for (void *p : c->csr_owned) cudaFree(p);
    for (void *p : c->pk_owned) cudaFree(p);
    for (void *p : c->pkt_owned) cudaFree(p);
    if (c->h_desc) cudaFreeHost(c->h_desc);
    if (c->h_vbeb) cudaFreeHost(c->h_vbeb);
    if (c->l2_limit_set) cudaCtxResetPersistingL2Cache();
    if (c->have_ev)
        for (int i = 0; i < kNumEv; ++i) cudaEventDestroy(c->ev[i]);
    if (c->h_counters) cudaFreeHost(c->h_counters);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->stream2) {
        cudaStreamSynchronize(c->stream2);
        cudaStreamDestroy(c->stream2);
    }
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    for (int k = 0; k < kUpChunks; ++k)
        if (c->ev_up[k]) cudaEventDestroy(c->ev_up[k]);
    if (c->scan_tmp) cudaFree(c->scan_tmp);
    for (void *p : c->rv_owned) cudaFree(p);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return ISPAN_OK;
}

int ispan_ctx_set_stream(ispan_ctx *c, void *stream) {
    if (!c) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    drop_graphs(c);
    return ISPAN_OK;
}

int ispan_ctx_set_tuning(ispan_ctx *c, const ispan_tuning *t) {
    if (!c) return ISPAN_ERR_ARG;
    if (t && (t->async_v < 0 || t->async_e < 0 || t->async_deg < 0 || t->bfs_ctas_per_sm < 0 || t->color_levels < 0 ||
              t->color_pivots < 0))
        return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    c->tuning = t ? *t : ispan_tuning{0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    c->g_coop_w = 0;  // recompute the persistent grids
    drop_graphs(c);   // the captured graph holds the old values
    return ISPAN_OK;
}

int ispan_ctx_get_tuning(ispan_ctx *c, ispan_tuning *t) {
    if (!c || !t) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    t->async_v = c->tuning.async_v > 0 ? c->tuning.async_v : kAsyncV;
    t->async_e = c->tuning.async_e > 0 ? c->tuning.async_e : kAsyncE;
    t->async_deg = c->tuning.async_deg > 0 ? c->tuning.async_deg : kAsyncDeg;
    t->bfs_ctas_per_sm = c->tuning.bfs_ctas_per_sm;
    t->color_levels = c->tuning.color_levels > 0 ? c->tuning.color_levels : kCLevels;
    t->color_pivots = c->tuning.color_pivots > 0 ? c->tuning.color_pivots : kCPivots;
    t->color_compact = c->tuning.color_compact >= 0 ? 1 : -1;
    t->pair_searches = c->tuning.pair_searches;
    t->tiny_residual = c->tuning.tiny_residual > 0 ? 1 : -1;
    t->pdl = c->tuning.pdl >= 0 ? 1 : -1;
    return ISPAN_OK;
}

int ispan_scc_run(ispan_ctx *c, const ispan_csr *g, const ispan_params *p, int32_t *labels_out,
                  ispan_stats *st) {
    return run_common(c, g, 1, nullptr, p, labels_out, st);
}

int ispan_scc_run_batch(ispan_ctx *c, const ispan_csr *g, int32_t nseg, const int64_t *vbase,
                        const ispan_params *p, int32_t *labels_out, ispan_stats *st) {
    if (!vbase) return ISPAN_ERR_ARG;
    return run_common(c, g, nseg, vbase, p, labels_out, st);
}

int ispan_scc_run_graphs(ispan_ctx *c, const ispan_csr *gs, int32_t n, int32_t *const *labels_out,
                         const ispan_params *p, ispan_stats *st) {
    if (!c || !gs || n < 1 || !labels_out) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return ISPAN_ERR_CUDA;
    return run_graphs(c, gs, n, labels_out, p, st);
}

int ispan_graphs_pack(ispan_ctx *c, const ispan_csr *gs, int32_t n) {
    if (!c || !gs || n < 1) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return ISPAN_ERR_CUDA;
    return pack_graphs(c, gs, n);
}

int ispan_graphs_run(ispan_ctx *c, const ispan_csr *gs, int32_t n, int32_t *const *labels_out,
                     const ispan_params *p, ispan_stats *st) {
    if (!c || !gs || n < 1 || !labels_out) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return ISPAN_ERR_CUDA;
    return run_packed(c, gs, n, labels_out, p, st);
}

int ispan_ref_codes(ispan_ctx *c, int32_t *codes) {
    if (!c || !codes) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    int64_t V = c->last_V;
    std::vector<int32_t> lab(V);
    std::vector<uint8_t> cls(V);
    std::vector<uint32_t> tm((V + 31) / 32 + 1), bm((V + 31) / 32 + 1);
    if (V) {
        CK(cudaMemcpy(lab.data(), c->last_label, V * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(cls.data(), c->cls, V, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(tm.data(), c->T, ((V + 31) / 32) * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(bm.data(), c->B, ((V + 31) / 32) * 4, cudaMemcpyDeviceToHost));
    }
    for (int64_t v = 0; v < V; ++v) {
        // the giant and the first trim are recorded as bitmaps, later classes per vertex
        uint8_t k = ((bm[v >> 5] >> (v & 31)) & 1u) ? (uint8_t)CLS_GIANT
                    : ((tm[v >> 5] >> (v & 31)) & 1u) ? (uint8_t)CLS_TRIM1 : cls[v];
        switch (k) {
            case CLS_GIANT: codes[v] = 1; break;
            case CLS_TRIM1: codes[v] = -1; break;
            case CLS_TRIM2: codes[v] = -2; break;
            case CLS_TRIM3: codes[v] = -3; break;
            default: codes[v] = lab[v] + 2; break;
        }
    }
    codes[V] = 0;
    return ISPAN_OK;
}

int ispan_debug_barrier_timeout(ispan_ctx *c, int64_t limit_us) {
    if (!c || limit_us <= 0 || limit_us > 10 * 1000 * 1000) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return ISPAN_ERR_CUDA;
    CK(cudaMemsetAsync(c->gsync, 0, kGridSyncWords * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->err, 0, 4 * sizeof(int), c->stream));
    k_barrier_probe<<<2, 32, 0, c->stream>>>(c->gsync, c->err, (uint64_t)limit_us * 1000ull);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_err, c->err, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const int e = c->h_err[0];
    // leave the barrier state clean for the next run (runs reset it too)
    CK(cudaMemsetAsync(c->gsync, 0, kGridSyncWords * sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->err, 0, 4 * sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return e;
}

int ispan_debug_trace(ispan_ctx *c, int64_t *out, int64_t cap) {
    if (!c || !out) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lock(c->mu);
    int64_t n = std::min<int64_t>(cap, 4 * kTraceLevels * 4);
    CK(cudaMemcpy(out, c->trace, n * sizeof(int64_t), cudaMemcpyDeviceToHost));
    return ISPAN_OK;
}

const char *ispan_strerror(int code) {
    switch (code) {
        case ISPAN_OK: return "ok";
        case ISPAN_ERR_ARG: return "bad argument or malformed CSR";
        case ISPAN_ERR_NOMEM: return "device allocation failed";
        case ISPAN_ERR_CUDA: return "CUDA runtime error";
        case ISPAN_ERR_TIMEOUT: return "device-side wait timed out";
        case ISPAN_ERR_INTERNAL: return "internal device-side check failed";
        case ISPAN_ERR_NODEV: return "no CUDA device";
        case ISPAN_ERR_CAPACITY: return "graph exceeds the context's capacity";
        case ISPAN_ERR_BUSY: return "request queue full";
        default: return "unknown error";
    }
}

const char *ispan_version(void) { return "ispan_b200 0.1 (sm_100a)"; }

}  // extern "C"

// stages.cuh -- every stage of the pipeline except the reachability
// searches (bfs.cuh).  Each kernel cites the reference function it replaces.
//
// Soundness of the concurrent trims: a trim kernel claims a vertex set only
// when the set is strongly connected through static edges and closed (in one
// edge direction) over the vertices it observed as still active.  Vertices
// only ever leave the active map, and only as whole true SCCs, so an
// observation "x is inactive" always means x belongs to another, already
// final SCC -- unless a concurrent claim of a *larger* set is in flight.
// Kernels therefore never mix claim sizes: trim-2 and trim-3 run as separate
// launches, and the peel (trim-1) decides from counters, not observations.
#pragma once
#include "common.cuh"

namespace ispan {

// classes recorded per vertex (for the reference-convention codes)
enum Cls : uint8_t { CLS_NONE = 0, CLS_GIANT = 1, CLS_TRIM1 = 2, CLS_TRIM2 = 3, CLS_TRIM3 = 4, CLS_MICE = 5 };

// control-block slots (Run::ctl64): worklist and queue counters
enum Ctl64 {
    K_WL0 = 0, K_WL1, K_CQ0, K_CQ1, K_CQ2, K_ROOTS, K_SMALL, K_LARGE, K_ALLOC, K_LARGE2,
    K_SPILL, K_MICE_SCC, K_LOCAL_NEXT, K_MINPRIO0, K_MINPRIO1, K_CAND,
    K_CMP_OK, K_CMP_EF, K_CMP_EB,  // compact colouring graph: built (1), its edge counts
    K_WCC_GIANT,                   // (root << 32) | 1 when one WCC holds half the root sample
    K_TINY,                        // 1: k_tiny_residual solved the residual; later stages return at once
    kNumCtl = 32
};

constexpr int kLocalV = 1024;   // a WCC up to this many vertices ...
constexpr int kLocalE = 4096;   // ... and internal edges is solved in shared memory

template <typename OffT>
struct Ext {
    unsigned long long *ctl;      // [kNumCtl]
    int32_t *roots;               // [V] WCC roots
    int32_t *small;               // [V] small WCC roots
    int32_t *large[2];            // [V] vertices of large WCCs (double buffered)
    int32_t *cq[2];               // [V] peel cascade queues
    int32_t *cand;                // [V] trim-2/3 candidates left by the first peel (count K_CAND)
    const int32_t *old;           // colouring on the compact graph: original id of each compact id
                                  // (NULL: the colouring runs on the input graph's ids)
};

// original vertex id of a colouring vertex id
template <typename OffT>
__device__ __forceinline__ int32_t orig_id(const Ext<OffT> &x, int32_t v) {
    return x.old ? __ldg(x.old + v) : v;
}

// ---------------------------------------------------------------------------
// Block-level compaction of bitmap words into a worklist with one atomic per
// CTA: the CTA owns a contiguous range of words, counts, reserves, then
// writes its vertices in word order.
template <typename WordFn>
__device__ void compact_words(int64_t W, WordFn f, int32_t *out, unsigned long long *cnt) {
    __shared__ int64_t sh[kWarps];
    __shared__ int s_warp[kWarps];
    __shared__ unsigned long long s_base;
    const int warp = threadIdx.x >> 5, lane = lane_id();
    int64_t per = (W + gridDim.x - 1) / gridDim.x;
    int64_t w0 = min(W, (int64_t)blockIdx.x * per), w1 = min(W, w0 + per);
    int64_t mine = 0;
    for (int64_t wi = w0 + threadIdx.x; wi < w1; wi += kBlock) mine += __popc(f(wi));
    int64_t tot = block_sum64(mine, sh);
    if (threadIdx.x == 0) s_base = tot ? atomicAdd(cnt, (unsigned long long)tot) : 0;
    __syncthreads();
    int64_t run = (int64_t)s_base;
    for (int64_t wb = w0; wb < w1; wb += kWarps) {
        int64_t wi = wb + warp;
        uint32_t m = (wi < w1) ? f(wi) : 0u;  // every lane evaluates; same value
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        int off = 0, all = 0;
        for (int i = 0; i < kWarps; ++i) {
            if (i < warp) off += s_warp[i];
            all += s_warp[i];
        }
        if ((m >> lane) & 1u) {
            int64_t at = run + off + __popc(m & lanemask_lt());
            if (VOK(at, 13)) out[at] = (int32_t)(wi * 32 + lane);
        }
        run += all;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Per-run reset: zero the run's counters, histogram, barrier and error
// words, trace and per-graph tables, and set the per-graph giant minima to
// "none", in one launch (each range a multiple of 4 bytes).
struct ResetRange { void *p; int64_t bytes; };
struct ResetDesc {
    ResetRange z[7];
    int32_t *gmin;
    int64_t nseg;
};

__global__ void k_reset(ResetDesc d) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nt = (int64_t)gridDim.x * blockDim.x;
#pragma unroll 1
    for (int k = 0; k < 7; ++k) {
        uint32_t *p = reinterpret_cast<uint32_t *>(d.z[k].p);
        const int64_t n = d.z[k].bytes / 4;
        for (int64_t i = gt; i < n; i += nt) p[i] = 0u;
    }
    for (int64_t i = gt; i < d.nseg; i += nt) d.gmin[i] = 0x7f7f7f7f;
}

// ---------------------------------------------------------------------------
// Input check on the device: offsets monotone from 0 to E, every adjacency
// id in [0, V).  The reference's loader trusts its files (src/graph.cpp:2-92);
// here a malformed CSR is reported as ISPAN_ERR_ARG before any stage reads it.
template <typename OffT>
__global__ void k_validate(const OffT *fb, const OffT *bb, const int32_t *fa, const int32_t *ba, int64_t V,
                           int64_t E, int *bad) {
    const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x, nt = (int64_t)gridDim.x * blockDim.x;
    int err = 0;
    for (int64_t i = gt; i <= V; i += nt) {
        int64_t a = fb[i], b = bb[i];
        if (i == 0 && (a != 0 || b != 0)) err = 1;
        if (i == V && (a != E || b != E)) err = 1;
        if (i < V && (fb[i + 1] < a || bb[i + 1] < b)) err = 1;
    }
    for (int64_t e = gt; e < E; e += nt) {
        int32_t x = fa[e], y = ba[e];
        if (x < 0 || x >= V || y < 0 || y >= V) err = 1;
    }
    if (__syncthreads_or(err) && threadIdx.x == 0) atomicExch(bad, 1);
}

// ---------------------------------------------------------------------------
// trim_1_first (src/trim_1_gfq.h:9-33) fused with generate_frontier_queue's
// bookkeeping (:486-529) and pivot_selection_from_fq (src/scc_common.h:92-150):
// one pass over the offsets.  A vertex with zero full out- or in-degree is its
// own SCC; the rest form the active map.  Pivot key per graph:
// (min(outdeg*indeg, 2^32-1) << 32) | ~id, i.e. the largest degree product,
// ties to the lowest id, in 64-bit arithmetic (the reference's int32 product
// overflows on hubs).
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_trim1_first(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    constexpr int U = 4;  // words per warp step: four independent offset loads in flight
    const int lane = lane_id();
    const int64_t gw = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int64_t nw = (int64_t)gridDim.x * kWarps;
    int64_t n_act = 0, mu = 0, mui = 0, n_tr = 0;
    unsigned long long best = 0;
    for (int64_t wb = gw * U; wb < r.W; wb += nw * U) {
        int64_t od[U], id[U];
        bool valid[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const int64_t v = (wb + j) * 32 + lane;
            valid[j] = (wb + j) < r.W && v < r.V;
            od[j] = valid[j] ? ld_off(r.fw_beg, v + 1) - ld_off(r.fw_beg, v) : 0;
            id[j] = valid[j] ? ld_off(r.bw_beg, v + 1) - ld_off(r.bw_beg, v) : 0;
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const int64_t wi = wb + j;
            const int64_t v = wi * 32 + lane;
            const bool act = valid[j] && od[j] > 0 && id[j] > 0;
            const unsigned am = __ballot_sync(kFull, act);
            const unsigned tm = __ballot_sync(kFull, valid[j] && !act);
            if (lane == 0 && wi < r.W) {
                r.A[wi] = am;
                r.T[wi] = tm;  // size-1 SCCs of the first trim; labelled by k_finalize
                r.F[wi] = 0;
                r.B[wi] = 0;
                r.D[wi] = 0;
            }
            n_tr += valid[j] && !act;
            unsigned long long key = 0;
            if (act) {
                ++n_act;
                mu += od[j];
                mui += id[j];
                unsigned long long prod = (unsigned long long)od[j] * (unsigned long long)id[j];
                if (prod > 0xffffffffull) prod = 0xffffffffull;
                key = (prod << 32) | (0xffffffffull - (unsigned long long)v);
            }
            if (r.nseg == 1) {
                best = key > best ? key : best;
            } else if (__any_sync(kFull, key != 0)) {
                // segmented: graphs are contiguous id ranges, so the word's first
                // and last vertex decide whether all lanes share one graph
                const int64_t vl = min(wi * 32 + 31, r.V - 1);
                int s0 = 0, s1 = 0;
                if (lane == 0) { s0 = seg_of(r.vbase, r.nseg, wi * 32); s1 = seg_of(r.vbase, r.nseg, vl); }
                s0 = __shfl_sync(kFull, s0, 0);
                s1 = __shfl_sync(kFull, s1, 0);
                if (s0 == s1) {
                    unsigned long long m = warp_max_u64(key);
                    if (lane == 0 && m) atomicMax(r.pivot_key + s0, m);
                } else if (key) {
                    atomicMax(r.pivot_key + seg_of(r.vbase, r.nseg, v), key);
                }
            }
        }
    }
    if (r.nseg == 1) {
        best = warp_max_u64(best);
        if (lane == 0 && best) atomicMax(r.pivot_key, best);
    }
    int64_t a = block_sum64(n_act, sh), m = block_sum64(mu, sh), mi = block_sum64(mui, sh), t = block_sum64(n_tr, sh);
    if (threadIdx.x == 0) {
        if (a) atomicAdd(r.counters + C_ACTIVE0, (unsigned long long)a);
        if (m) atomicAdd(r.counters + C_MU0, (unsigned long long)m);
        if (mi) atomicAdd(r.counters + C_MU0_IN, (unsigned long long)mi);
        if (t) atomicAdd(r.counters + C_TRIM1, (unsigned long long)t);
    }
}

// Seed the forward (DIR 0) or backward (DIR 1) search with each graph's
// pivot: mark it, queue it at level 0.  Warp per 32 graphs.
template <typename OffT, int DIR>
__global__ void k_seed(Run<OffT> r) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    const int lane = lane_id();
    int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int64_t nwp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t b = gw * 32; b < r.nseg; b += nwp * 32) {
        int64_t s = b + lane;
        unsigned long long key = s < r.nseg ? r.pivot_key[s] : 0ull;
        bool ok = key != 0;
        int64_t p = ok ? (int64_t)(0xffffffffull - (key & 0xffffffffull)) : 0;
        int64_t dg = 0;
        if (ok) {
            if (DIR == 0) {
                set_bit(r.F, p);
                dg = ld_off(r.fw_beg, p + 1) - ld_off(r.fw_beg, p);
                atomicAdd(r.counters + C_FW_SIZE, 1ull);
            } else {
                set_bit(r.B, p);
                dg = ld_off(r.bw_beg, p + 1) - ld_off(r.bw_beg, p);
            }
        }
        q_append(ok, (int32_t)p, dg, r.qv[0], r.qe[0], r.qchunk[0], r.qpk, r.V);
    }
}

// The pivot SCC of each graph is B (reached backward inside F; F & B when
// the searches ran at the same time).  One pass
// over the maps: B leaves the active map, each graph's minimum member id (its
// canonical label, written by k_finalize) and size are taken, and the
// remaining active vertices are compacted into the residual worklist.  Each
// CTA owns a contiguous range of words, one word per thread per step; one
// atomic per CTA reserves its share of the worklist.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_giant_residual(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    __shared__ int s_scan[kWarps];
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x, lane = lane_id(), warp = tid >> 5;
    const int64_t per = (r.W + gridDim.x - 1) / gridDim.x;
    const int64_t w0 = min(r.W, (int64_t)blockIdx.x * per), w1 = min(r.W, w0 + per);
    int64_t n_giant = 0, n_res = 0;
    int gm = 0x7fffffff;
    // pass 1: update A, giant stats, count the residual
    const bool pair = (r.flags & kRunPair) != 0;
    for (int64_t wi = w0 + tid; wi < w1; wi += kBlock) {
        uint32_t a = r.A[wi], b = r.B[wi];
        if (pair) {  // the backward search ran over A: the pivot SCC is F & B; D held its snapshots
            b &= r.F[wi];
            r.B[wi] = b;
            r.D[wi] = 0u;
        }
        uint32_t res = a & ~b;
        if (b) r.A[wi] = res;
        n_res += __popc(res);
        if (b) {
            n_giant += __popc(b);
            int v0 = (int)(wi * 32 + __ffs(b) - 1);  // the word's smallest member
            if (r.nseg == 1) {
                gm = min(gm, v0);
            } else {
                const int64_t vlast = wi * 32 + 31 - __clz(b);
                const int sa = seg_of(r.vbase, r.nseg, v0), sb = seg_of(r.vbase, r.nseg, vlast);
                if (sa == sb) {  // graphs are contiguous ranges: one graph holds the whole word
                    atomicMin(r.gmin + sa, v0);
                    atomicAdd(r.gsize + sa, (unsigned long long)__popc(b));
                } else {
                    for (uint32_t m = b; m;) {  // the word straddles graphs
                        int bit = __ffs(m) - 1;
                        int64_t v = wi * 32 + bit;
                        int sg = seg_of(r.vbase, r.nseg, v);
                        atomicMin(r.gmin + sg, (int)v);
                        atomicAdd(r.gsize + sg, 1ull);
                        m &= m - 1;
                    }
                }
            }
        }
    }
    if (r.nseg == 1) {
        gm = warp_min(gm);
        if (lane == 0 && gm != 0x7fffffff) atomicMin(r.gmin, gm);
    }
    int64_t tg = block_sum64(n_giant, sh), tr = block_sum64(n_res, sh);
    if (tid == 0) {
        if (tg) {
            atomicAdd(r.counters + C_GIANT, (unsigned long long)tg);
            if (r.nseg == 1) atomicAdd(r.gsize, (unsigned long long)tg);
        }
        s_base = tr ? atomicAdd(x.ctl + K_WL0, (unsigned long long)tr) : 0ull;
    }
    __syncthreads();
    // pass 2: write the residual vertices in word order
    int64_t run = (int64_t)s_base;
    for (int64_t wb = w0; wb < w1; wb += kBlock) {
        int64_t wi = wb + tid;
        uint32_t m = wi < w1 ? __ldcg(r.A + wi) : 0u;
        int c = __popc(m), incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_scan[warp] = incl;
        __syncthreads();
        int off = 0, all = 0;
#pragma unroll
        for (int i = 0; i < kWarps; ++i) {
            int t = s_scan[i];
            off += i < warp ? t : 0;
            all += t;
        }
        int64_t at = run + off + incl - c;
        for (; m; m &= m - 1) {
            if (VOK(at, 13)) r.wl[0][at] = (int32_t)(wi * 32 + __ffs(m) - 1);
            ++at;
        }
        run += all;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// trim_1_from_fq_gfq (src/trim_1_gfq.h:365-458) and its loops
// (src/scc_core.cpp:562-602, :757-795), run to a fixpoint in one persistent
// kernel: count each worklist vertex's active non-self in/out edges once,
// then peel with a cascade -- a vertex whose last active out- (or in-)
// neighbour is peeled reaches a zero counter and is peeled in the next round.
// Work is proportional to the edges of the peeled vertices, not to
// (passes x residual edges).  Survivors are compacted into the other worklist.
template <typename OffT>
__device__ __forceinline__ void count_active(const OffT *beg, const int32_t *adj, const uint32_t *A, int64_t v,
                                             int32_t &n) {
    int64_t e0 = ld_off(beg, v), e1 = ld_off(beg, v + 1);
    int c = 0;
    // four ids, then their active bits, each group of loads in flight together
    for (int64_t e = e0; e < e1; e += 4) {
        int32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = e + q < e1 ? ld_adj(adj, e + q) : (int32_t)v;
#pragma unroll
        for (int q = 0; q < 4; ++q) c += (w[q] != v) && bitc(A, w[q]);
    }
    n = c;
}

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_trim1(Run<OffT> r, Ext<OffT> x, int in, int out, int cand) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    __shared__ int64_t sh[kWarps];
    const int64_t gt = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    const int64_t nt = (int64_t)gridDim.x * kBlock;
    const int32_t *wl = r.wl[in];
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    unsigned long long *cqc = x.ctl + K_CQ0;  // 3 rotating counters
    if (n == 0) {  // every CTA reads the same count: no barrier needed to leave
        if (cand && blockIdx.x == 0 && threadIdx.x == 0) {
            x.ctl[K_WL0 + in] = 0ull;
            cqc[0] = cqc[1] = cqc[2] = 0ull;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(r.counters + C_TRIM_ROUNDS, 1ull);
        return;
    }
    // phase 1: counts against the active map as it stands (nothing is
    // cleared until the barrier, so the counts are exact)
    for (int64_t i = gt; i - (threadIdx.x) < n; i += nt) {
        bool dead = false;
        int32_t v = 0;
        if (i < n) {
            v = wl[i];
            if (bitc(r.A, v)) {
                int32_t o, ii;
                count_active(r.fw_beg, r.fw_adj, r.A, v, o);
                count_active(r.bw_beg, r.bw_adj, r.A, v, ii);  // independent of o: both in flight
                if (o == 0 || ii == 0) {
                    dead = set_bit(r.D, v);
                } else {
                    r.cnt_out[v] = o;
                    r.cnt_in[v] = ii;
                }
            }
        }
        wl_append(dead, v, x.cq[0], cqc + 0);
    }
    if (!grid_sync(r.gsync, r.err)) return;
    // every CTA has read the list count: with `cand` (the first peel) it is
    // cleared for the second peel, which appends its survivors there
    if (cand && blockIdx.x == 0 && threadIdx.x == 0) x.ctl[K_WL0 + in] = 0ull;
    // cascade rounds
    int lv = 0;
    for (int guard = 0; guard < (1 << 30); ++guard) {
        const int c = lv & 1;
        const int64_t m = (int64_t)__ldcg(cqc + lv % 3);
        if (m == 0) {
            // every CTA reads this zero slot; the other two are free, and the
            // second peel starts its cascade from three zero counters
            if (cand && blockIdx.x == 0 && threadIdx.x == 0) { cqc[(lv + 1) % 3] = 0ull; cqc[(lv + 2) % 3] = 0ull; }
            break;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) cqc[(lv + 2) % 3] = 0ull;
        const int32_t *q = x.cq[c];
        for (int64_t i = gt; i - threadIdx.x < m; i += nt) {
            int32_t t = i < m ? __ldcg(q + i) : 0;
            bool live = i < m;
            // out-edges t->w lower w's in-count; in-edges u->t lower u's out-count
            for (int dir = 0; dir < 2; ++dir) {
                const OffT *beg = dir == 0 ? r.fw_beg : r.bw_beg;
                const int32_t *adj = dir == 0 ? r.fw_adj : r.bw_adj;
                int32_t *cnt = dir == 0 ? r.cnt_in : r.cnt_out;
                int64_t e0 = live ? ld_off(beg, t) : 0, e1 = live ? ld_off(beg, t + 1) : 0;
                // edges one by one; appends are warp-aggregated per step
                int64_t len = e1 - e0;
                int64_t maxlen = len;
                for (int o = 16; o; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(kFull, maxlen, o));
                for (int64_t k = 0; k < maxlen; ++k) {
                    bool nd = false;
                    int32_t w = 0;
                    if (k < len) {
                        w = ld_adj(adj, e0 + k);
                        if (w != t && bitc(r.A, w) && !bitv(r.D, w)) {
                            if (atomicSub(cnt + w, 1) == 1) nd = set_bit(r.D, w);
                        }
                    }
                    wl_append(nd, w, x.cq[c ^ 1], cqc + (lv + 1) % 3);
                }
            }
        }
        if (!grid_sync(r.gsync, r.err)) return;
        ++lv;
    }
    // final: peeled vertices leave; survivors move to the other worklist.
    // With `cand` set, survivors with at most two active out- or in-edges
    // (the counters are exact after the cascade) are also listed as the
    // trim-2/3 candidates: every vertex of a 2- or 3-vertex pattern has at
    // most two distinct active successors (or predecessors), so without
    // duplicate edges no pattern is missed; with duplicates a pattern may be
    // left to the later stages, which find the same SCC.
    int64_t peeled = 0;
    for (int64_t i = gt; i - threadIdx.x < n; i += nt) {
        bool keep = false, cd = false;
        int32_t v = 0;
        if (i < n) {
            v = wl[i];
            if (bitc(r.A, v)) {
                if (bitv(r.D, v)) {
                    clear_bit(r.A, v);
                    r.label[v] = v;
                    r.cls[v] = CLS_TRIM1;
                    ++peeled;
                } else {
                    keep = true;
                    cd = cand && (__ldcg(r.cnt_out + v) <= 2 || __ldcg(r.cnt_in + v) <= 2);
                }
            }
        }
        wl_append(keep, v, r.wl[out], x.ctl + K_WL0 + out);
        if (cand) wl_append(cd, v, x.cand, x.ctl + K_CAND);
    }
    int64_t tp = block_sum64(peeled, sh);
    if (threadIdx.x == 0) {
        if (tp) atomicAdd(r.counters + C_TRIM1, (unsigned long long)tp);
        if (blockIdx.x == 0) atomicAdd(r.counters + C_TRIM_ROUNDS, (unsigned long long)(lv + 1));
    }
}

// ---------------------------------------------------------------------------
// trim-2 / trim-3 pattern checks.  distinct_active: up to `cap` distinct
// active neighbours of v in one direction, skipping x1 and x2.
template <typename OffT>
__device__ __forceinline__ int distinct_active(const OffT *beg, const int32_t *adj, const uint32_t *A, int64_t v,
                                               int32_t x1, int32_t x2, int cap, int32_t &n1, int32_t &n2) {
    int64_t e0 = ld_off(beg, v), e1 = ld_off(beg, v + 1);
    int d = 0;
    // four edges per step: their ids, then their active bits, each group of
    // loads in flight together; the early exit stays per edge
    for (int64_t e = e0; e < e1 && d < cap; e += 4) {
        int32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = e + q < e1 ? ld_adj(adj, e + q) : -1;
        bool act[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) act[q] = w[q] >= 0 && w[q] != x1 && w[q] != x2 && bitv(A, w[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (!act[q] || d >= cap) continue;
            if (d == 0) { n1 = w[q]; d = 1; }
            else if (d == 1 && w[q] != n1) { n2 = w[q]; d = 2; }
            else if (d == 2 && w[q] != n1 && w[q] != n2) { d = 3; }
        }
    }
    return d;
}

template <typename OffT>
__device__ __forceinline__ bool claim(Run<OffT> &r, Ext<OffT> &x, int32_t v, int32_t lab, uint8_t cls) {
    if (!set_bit(r.D, v)) return false;
    r.label[v] = lab;
    r.cls[v] = cls;
    clear_bit(r.A, v);
    return true;
}

// trim_2_from_fq (src/trim_2_3.h:146-283): sink 2-cycles (the vertex's only
// active successor has the vertex as its only active successor) and source
// 2-cycles (the same over predecessors).  Label = min of the pair.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_trim2(Run<OffT> r, Ext<OffT> x, const int32_t *wl,
                                                  const unsigned long long *n_wl) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    __shared__ int64_t sh[kWarps];
    const int64_t n = (int64_t)__ldcg(n_wl);
    int64_t got = 0;
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        int32_t v = wl[i];
        if (!bitv(r.A, v)) continue;
        for (int dir = 0; dir < 2; ++dir) {
            const OffT *beg = dir == 0 ? r.fw_beg : r.bw_beg;
            const int32_t *adj = dir == 0 ? r.fw_adj : r.bw_adj;
            int32_t a = -1, b = -1, c = -1, dd = -1;
            if (distinct_active(beg, adj, r.A, v, v, v, 2, a, b) != 1) continue;
            if (distinct_active(beg, adj, r.A, a, a, a, 2, c, dd) != 1 || c != v) continue;
            int32_t lab = min(v, a);
            got += claim(r, x, v, lab, CLS_TRIM2);
            got += claim(r, x, a, lab, CLS_TRIM2);
            break;
        }
    }
    int64_t t = block_sum64(got, sh);
    if (threadIdx.x == 0 && t) atomicAdd(r.counters + C_TRIM2, (unsigned long long)t);
}

// trim_3_1_from_fq (src/trim_2_3.h:482-677, cycle A->B->C->A) and
// trim_3_2_from_fq (:881-1080, hub A<->B, A<->C) in one launch: both claim
// 3-vertex sets, so they may run concurrently.  Label = min of the three.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_trim3(Run<OffT> r, Ext<OffT> x, const int32_t *wl,
                                                  const unsigned long long *n_wl) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    __shared__ int64_t sh[kWarps];
    const int64_t n = (int64_t)__ldcg(n_wl);
    int64_t got = 0;
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        int32_t v = wl[i];
        if (!bitv(r.A, v)) continue;
        for (int dir = 0; dir < 2; ++dir) {
            const OffT *beg = dir == 0 ? r.fw_beg : r.bw_beg;
            const int32_t *adj = dir == 0 ? r.fw_adj : r.bw_adj;
            int32_t B = -1, C = -1, y = -1, z = -1;
            int nv = distinct_active(beg, adj, r.A, v, v, v, 3, B, C);
            int32_t m0 = -1, m1 = -1, m2 = -1;
            if (nv == 1) {  // cycle shape: v -> B -> C -> v
                if (distinct_active(beg, adj, r.A, B, B, v, 2, y, z) != 1) continue;
                int32_t Cc = y;
                if (distinct_active(beg, adj, r.A, Cc, Cc, B, 2, y, z) != 1 || y != v) continue;
                m0 = v; m1 = B; m2 = Cc;
            } else if (nv == 2) {  // hub shape: v <-> B, v <-> C
                if (distinct_active(beg, adj, r.A, B, B, C, 2, y, z) != 1 || y != v) continue;
                if (distinct_active(beg, adj, r.A, C, C, B, 2, y, z) != 1 || y != v) continue;
                m0 = v; m1 = B; m2 = C;
            } else {
                continue;
            }
            int32_t lab = min(m0, min(m1, m2));
            got += claim(r, x, m0, lab, CLS_TRIM3);
            got += claim(r, x, m1, lab, CLS_TRIM3);
            got += claim(r, x, m2, lab, CLS_TRIM3);
            break;
        }
    }
    int64_t t = block_sum64(got, sh);
    if (threadIdx.x == 0 && t) atomicAdd(r.counters + C_TRIM3, (unsigned long long)t);
}

// ---------------------------------------------------------------------------
// Weakly connected components of the residual: hook-and-pointer-jump
// union-find (replaces coloring_wcc, src/color_propagation.h:468-593, and the
// unused openmp_wcc, src/openmp_wcc.hpp:14-165).  Roots are hooked under the
// smaller id, so every root is its component's minimum vertex and parent ids
// strictly decrease along a path; path halving keeps that invariant.
__device__ __forceinline__ int32_t uf_find(int32_t *parent, int32_t x) {
    int32_t p = __ldcg(parent + x);
    while (p != x) {
        int32_t gp = __ldcg(parent + p);
        if (gp != p) parent[x] = gp;  // halving; gp < p < x
        x = p;
        p = gp;
    }
    return x;
}

// Read-only root walk for the flatten pass: once hooking is over, path
// halving must not run concurrently with the final `parent[v] = root` writes,
// or a halving store could replace a final root with an intermediate ancestor.
__device__ __forceinline__ int32_t uf_root(const int32_t *parent, int32_t x) {
    int32_t p = __ldcg(parent + x);
    while (p != x) {
        x = p;
        p = __ldcg(parent + x);
    }
    return x;
}

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_init(Run<OffT> r, Ext<OffT> x, int in) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        int32_t v = r.wl[in][i];
        r.parent[v] = v;
        r.aux[v] = 0;      // member count (valid at roots)
        r.aux2[v] = -1;    // member base of a small WCC
        r.cnt_out[v] = 0;  // fill cursor
    }
    // a batch's per-graph giant roots are marked in D (free after the peels)
    if (r.nseg > 1)
        for (int64_t w = (int64_t)blockIdx.x * kBlock + threadIdx.x; w < r.W; w += (int64_t)gridDim.x * kBlock)
            r.D[w] = 0u;
}

// hook the active neighbours adj[e0, e1) of v (four ids, then their active
// bits, in flight together)
__device__ __forceinline__ void hook_range(int32_t *parent, const uint32_t *A, const int32_t *adj, int32_t v,
                                           int64_t e0, int64_t e1) {
    for (int64_t e = e0; e < e1; e += 4) {
        int32_t ws[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) ws[q] = e + q < e1 ? ld_adj(adj, e + q) : v;
        bool act[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) act[q] = ws[q] != v && bitc(A, ws[q]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (!act[q]) continue;
            int32_t a = v, b = ws[q];
            for (int guard = 0; guard < (1 << 20); ++guard) {
                a = uf_find(parent, a);
                b = uf_find(parent, b);
                if (a == b) break;
                if (a > b) { int32_t t = a; a = b; b = t; }
                int32_t old = atomicCAS(parent + b, b, a);  // hook root b under a
                if (old == b) break;
                b = old;
            }
        }
    }
}

// Hooking in the manner of Afforest (neighbour sampling): phase 0 links
// every vertex with its first kWccSample out-neighbours; after a compress
// pass and a sample of the roots, phase 1 links the rest.  When one
// component holds at least half of the sample (a giant WCC), its members
// skip phase 1: every edge with an endpoint outside it is linked from that
// endpoint (its remaining out-edges and all its in-edges), and edges inside
// it are already connected.  Otherwise every vertex links its remaining
// out-edges.
constexpr int kWccSample = 2;
constexpr int kWccRootSamples = 512;
constexpr int64_t kWccSkipMin = 1 << 14;  // smaller worklists: no sample, everyone links everything

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_hook(Run<OffT> r, Ext<OffT> x, int in, int phase) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    const bool skip_giant = phase == 1 && (r.nseg > 1 || __ldcg(x.ctl + K_WCC_GIANT) != 0);
    const int32_t g = (int32_t)(__ldcg(x.ctl + K_WCC_GIANT) >> 32);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        int32_t v = r.wl[in][i];
        const int64_t e0 = ld_off(r.fw_beg, v), e1 = ld_off(r.fw_beg, v + 1);
        const int64_t es = min(e1, e0 + kWccSample);
        if (phase == 0) {
            hook_range(r.parent, r.A, r.fw_adj, v, e0, es);
        } else if (!skip_giant) {
            hook_range(r.parent, r.A, r.fw_adj, v, es, e1);
        } else {
            // outside its graph's giant WCC (one graph: the sampled root g;
            // a batch: roots marked in D by k_wcc_giant_seg), link both ways
            const int32_t pv = __ldcg(r.parent + v);
            if (r.nseg > 1 ? !bitc(r.D, pv) : pv != g) {
                hook_range(r.parent, r.A, r.fw_adj, v, es, e1);
                hook_range(r.parent, r.A, r.bw_adj, v, ld_off(r.bw_beg, v), ld_off(r.bw_beg, v + 1));
            }
        }
    }
}

// after phase 0: every vertex points at its root (read-only walks; no hook
// runs concurrently), then one CTA samples the roots of evenly spaced
// vertices and records the most frequent one if it holds half the sample
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_compress(Run<OffT> r, Ext<OffT> x, int in) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        const int32_t v = r.wl[in][i];
        r.parent[v] = uf_root(r.parent, v);
    }
}

template <typename OffT>
__global__ void __launch_bounds__(kWccRootSamples) k_wcc_giant(Run<OffT> r, Ext<OffT> x, int in) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    __shared__ int32_t roots[kWccRootSamples];
    __shared__ int best, best_n;
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    const int t = threadIdx.x;
    if (n < kWccSkipMin) {  // (the reset left K_WCC_GIANT at zero)
        return;
    }
    const int ns = (int)(n < kWccRootSamples ? n : kWccRootSamples);
    if (t < ns) roots[t] = __ldcg(r.parent + r.wl[in][(int64_t)t * n / ns]);
    if (t == 0) { best = -1; best_n = 0; }
    __syncthreads();
    int cnt = 0;
    if (t < ns) {
        const int32_t me = roots[t];
        for (int k = 0; k < ns; ++k) cnt += roots[k] == me;
        atomicMax(&best_n, cnt);
    }
    __syncthreads();
    if (t < ns && cnt == best_n) atomicMax(&best, roots[t]);  // one root among the most frequent
    __syncthreads();
    if (t == 0)
        x.ctl[K_WCC_GIANT] = (ns > 0 && 2 * best_n >= ns) ? (((unsigned long long)(uint32_t)best << 32) | 1ull) : 0ull;
}

// The same for a batch, per graph: a warp samples 32 evenly spaced vertices
// of its graph's id range; among the active ones (the residual), a root
// held by at least half of them, and by at least two, is that graph's giant
// WCC and is marked in D.  Graphs never share a WCC, so no edge joins two
// marked components, and phase 1 links every edge with an endpoint outside
// them from that endpoint, as for one graph.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_giant_seg(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int lane = lane_id();
    const int64_t gw = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kBlock) >> 5;
    for (int64_t sg = gw; sg < r.nseg; sg += nw) {
        const int64_t v0 = r.vbase[sg], span = r.vbase[sg + 1] - v0;
        int32_t root = -1;
        if (span > 0) {
            const int64_t v = v0 + (int64_t)lane * span / 32;
            if ((lane < span || span >= 32) && bitc(r.A, v)) root = __ldcg(r.parent + v);
        }
        const unsigned act = __ballot_sync(kFull, root >= 0);
        const unsigned same = __match_any_sync(kFull, root);
        const int cnt = root >= 0 ? __popc(same & act) : 0;
        const int best = __reduce_max_sync(kFull, cnt);
        // the lowest lane holding the most frequent root decides
        const unsigned lead = __ballot_sync(kFull, cnt == best && best > 0);
        if (lane == __ffs(lead) - 1 && best >= 2 && 2 * best >= __popc(act)) set_bit(r.D, root);
    }
}

// flatten, count members per root, list the roots
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_flatten(Run<OffT> r, Ext<OffT> x, int in) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i - threadIdx.x < n;
         i += (int64_t)gridDim.x * kBlock) {
        bool isroot = false;
        int32_t v = 0;
        if (i < n) {
            v = r.wl[in][i];
            int32_t root = uf_root(r.parent, v);
            r.parent[v] = root;
            isroot = root == v;
            // warp-aggregate the member count per distinct root
            unsigned grp = __match_any_sync(__activemask(), root);
            if (lane_id() == __ffs(grp) - 1) atomicAdd(r.aux + root, __popc(grp));
        }
        wl_append(isroot, v, x.roots, x.ctl + K_ROOTS);
    }
}

// Reserve member space for small WCCs; route the rest to the large path.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_alloc(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int64_t n = (int64_t)__ldcg(x.ctl + K_ROOTS);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i - threadIdx.x < n;
         i += (int64_t)gridDim.x * kBlock) {
        bool sm = false;
        int32_t v = 0;
        if (i < n) {
            v = x.roots[i];
            int32_t c = r.aux[v];
            if (c <= kLocalV) {
                r.aux2[v] = (int32_t)atomicAdd(x.ctl + K_ALLOC, (unsigned long long)c);
                sm = true;
            }
        }
        wl_append(sm, v, x.small, x.ctl + K_SMALL);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(r.counters + C_WCC, (unsigned long long)n);
}

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_wcc_scatter(Run<OffT> r, Ext<OffT> x, int in) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    const int64_t n = (int64_t)__ldcg(x.ctl + K_WL0 + in);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i - threadIdx.x < n;
         i += (int64_t)gridDim.x * kBlock) {
        bool big = false;
        int32_t v = 0;
        if (i < n) {
            v = r.wl[in][i];
            int32_t root = r.parent[v];
            int32_t b = r.aux2[root];
            if (b >= 0) {
                int32_t k = atomicAdd(r.cnt_out + root, 1);
                if (VOK((long long)b + k, 15)) r.members[b + k] = v;
                r.cnt_in[v] = k;  // local index inside the WCC
            } else {
                big = true;
            }
        }
        wl_append(big, v, x.large[0], x.ctl + K_LARGE);
    }
}

// ---------------------------------------------------------------------------
// Small WCCs: one CTA per WCC builds the induced subgraph in shared memory
// and runs an iterative Tarjan on it (linear time; the reference's
// mice_fw_bw, src/fw_bw.h:1585-1691, runs one forward-backward search per
// pivot instead).  A WCC whose internal edges exceed kLocalE spills to the
// large (colouring) path.
constexpr int kLocalThreads = 256;

template <typename OffT>
__global__ void __launch_bounds__(kLocalThreads) k_local_scc(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (__ldcg(x.ctl + K_TINY)) return;  // the residual was solved in one CTA
    __shared__ int32_t gid[kLocalV];
    __shared__ int32_t loff[kLocalV + 1];
    __shared__ uint16_t ladj[kLocalE];
    __shared__ int16_t idx[kLocalV], low[kLocalV], stk[kLocalV], csv[kLocalV];
    __shared__ int32_t cse[kLocalV];
    __shared__ uint8_t onst[kLocalV];
    __shared__ uint32_t fwm[kLocalV / 32], bwm[kLocalV / 32], frm[2][kLocalV / 32];
    __shared__ int s_flag, s_min, s_both;
    __shared__ long long s_wq;
    const int64_t nsmall = (int64_t)__ldcg(x.ctl + K_SMALL);
    if (nsmall == 0) return;
    for (int guard = 0; guard < (1 << 30); ++guard) {
        // dynamic assignment: large and small WCCs interleave across CTAs
        __syncthreads();  // everyone is done with the previous WCC (and s_wq)
        if (threadIdx.x == 0) s_wq = (long long)atomicAdd(x.ctl + K_LOCAL_NEXT, 1ull);
        __syncthreads();
        const int64_t wq = s_wq;
        if (wq >= nsmall) break;
        const int32_t root = x.small[wq];
        const int32_t nv = r.aux[root];
        if (!ICHK(nv >= 1 && nv <= kLocalV, 17, nv)) continue;
        const int32_t base = r.aux2[root];
        // per-vertex internal out-degree, then a vertex-order scan by warp 0
        for (int i = threadIdx.x; i < nv; i += kLocalThreads) {
            int32_t u = r.members[base + i];
            gid[i] = u;
            int32_t dcount = 0;
            int64_t e0 = ld_off(r.fw_beg, u), e1 = ld_off(r.fw_beg, u + 1);
            for (int64_t e = e0; e < e1; ++e) {
                int32_t w = ld_adj(r.fw_adj, e);
                dcount += (w != u) && bitc(r.A, w);
            }
            loff[i + 1] = dcount;
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            int32_t carry = 0;
            if (threadIdx.x == 0) loff[0] = 0;
            for (int b0 = 0; b0 < nv; b0 += 32) {
                int i = b0 + threadIdx.x;
                int32_t inc = i < nv ? loff[i + 1] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    int32_t y = __shfl_up_sync(kFull, inc, o);
                    if (lane_id() >= o) inc += y;
                }
                if (i < nv) loff[i + 1] = carry + inc;
                carry += __shfl_sync(kFull, inc, 31);
            }
        }
        __syncthreads();
        const int32_t tot = loff[nv];
        if (tot > kLocalE) {
            // spill: hand the whole WCC to the colouring path
            for (int i = threadIdx.x; i < nv; i += kLocalThreads) {
                unsigned long long p = atomicAdd(x.ctl + K_LARGE, 1ull);
                if (VOK((long long)p, 16)) x.large[0][p] = gid[i];
            }
            if (threadIdx.x == 0) atomicAdd(r.counters + C_SPILL, 1ull);
            __syncthreads();
            continue;
        }
        // fill local adjacency (local ids from the scatter pass)
        for (int i = threadIdx.x; i < nv; i += kLocalThreads) {
            {
                int32_t u = gid[i];
                int32_t p = loff[i];
                int64_t e0 = ld_off(r.fw_beg, u), e1 = ld_off(r.fw_beg, u + 1);
                for (int64_t e = e0; e < e1; ++e) {
                    int32_t w = ld_adj(r.fw_adj, e);
                    if (w != u && bitc(r.A, w)) {
                        int32_t li = r.cnt_in[w];
                        if (ICHK(p < kLocalE && li >= 0 && li < nv, 14, ((long long)p << 32) | (li & 0xffffffff)))
                            ladj[p++] = (uint16_t)li;
                    }
                }
            }
        }
        __syncthreads();
        // One forward and one backward search from local vertex 0, all threads
        // on bitmaps in shared memory.  If both reach every vertex, the WCC is
        // a single SCC (the common case for planted cycles with chords) and
        // no serial work is needed.
        const int nw = (nv + 31) >> 5;
        for (int i = threadIdx.x; i < kLocalV / 32; i += kLocalThreads) {
            fwm[i] = 0; bwm[i] = 0; frm[0][i] = 0; frm[1][i] = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) { fwm[0] = 1u; frm[0][0] = 1u; bwm[0] = 1u; s_min = 0x7fffffff; }
        __syncthreads();
        for (int lv = 0, fc = 0; lv < kLocalV; ++lv, fc ^= 1) {  // forward, frontier push
            __syncthreads();  // all threads have read s_flag and frm of the last level
            if (threadIdx.x == 0) s_flag = 0;
            for (int i = threadIdx.x; i < kLocalV / 32; i += kLocalThreads) frm[fc ^ 1][i] = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < nv; i += kLocalThreads) {
                if (!((frm[fc][i >> 5] >> (i & 31)) & 1u)) continue;
                for (int e = loff[i]; e < loff[i + 1]; ++e) {
                    int w = ladj[e];
                    uint32_t bb = 1u << (w & 31);
                    if (!(atomicOr(&fwm[w >> 5], bb) & bb)) {
                        atomicOr(&frm[fc ^ 1][w >> 5], bb);
                        s_flag = 1;
                    }
                }
            }
            __syncthreads();
            if (!s_flag) break;
        }
        for (int lv = 0; lv < kLocalV; ++lv) {  // backward, pull over out-edges
            __syncthreads();
            if (threadIdx.x == 0) s_flag = 0;
            __syncthreads();
            for (int i = threadIdx.x; i < nv; i += kLocalThreads) {
                if ((bwm[i >> 5] >> (i & 31)) & 1u) continue;
                for (int e = loff[i]; e < loff[i + 1]; ++e)
                    if ((bwm[ladj[e] >> 5] >> (ladj[e] & 31)) & 1u) {
                        atomicOr(&bwm[i >> 5], 1u << (i & 31));
                        s_flag = 1;
                        break;
                    }
            }
            __syncthreads();
            if (!s_flag) break;
        }
        int both = 0;
        for (int i = threadIdx.x; i < nw; i += kLocalThreads) {
            uint32_t m = fwm[i] & bwm[i];
            if (i == nw - 1 && (nv & 31)) m &= (1u << (nv & 31)) - 1u;
            both += __popc(m);
        }
        for (int o = 16; o; o >>= 1) both += __shfl_xor_sync(kFull, both, o);
        __syncthreads();
        if (threadIdx.x == 0) s_both = 0;
        __syncthreads();
        if (lane_id() == 0) atomicAdd(&s_both, both);
        for (int i = threadIdx.x; i < nv; i += kLocalThreads) atomicMin(&s_min, gid[i]);
        __syncthreads();
        if (s_both == nv) {  // single SCC
            const int32_t mn = s_min;
            for (int i = threadIdx.x; i < nv; i += kLocalThreads) {
                r.label[gid[i]] = mn;
                r.cls[gid[i]] = CLS_MICE;
            }
            if (threadIdx.x == 0) {
                atomicAdd((unsigned long long *)(r.hist + nv), 1ull);  // nv <= kLocalV
                atomicAdd(r.counters + C_MICE_SCC, 1ull);
                atomicAdd(r.counters + C_MICE_V, (unsigned long long)nv);
                atomicAdd(r.counters + C_LOCAL_WCC, 1ull);
            }
        } else if (threadIdx.x == 0) {
            // iterative Tarjan over the local CSR
            for (int i = 0; i < nv; ++i) { idx[i] = -1; onst[i] = 0; }
            int counter = 0, sp = 0, nscc = 0;
            for (int s0 = 0; s0 < nv; ++s0) {
                if (idx[s0] != -1) continue;
                int cp = 0;
                csv[0] = (int16_t)s0; cse[0] = loff[s0]; cp = 1;
                idx[s0] = low[s0] = (int16_t)counter++;
                stk[sp++] = (int16_t)s0; onst[s0] = 1;
                while (cp > 0) {
                    int vv = csv[cp - 1];
                    int e = cse[cp - 1];
                    bool down = false;
                    for (; e < loff[vv + 1]; ++e) {
                        int w = ladj[e];
                        if (idx[w] == -1) {
                            cse[cp - 1] = e + 1;
                            idx[w] = low[w] = (int16_t)counter++;
                            stk[sp++] = (int16_t)w; onst[w] = 1;
                            csv[cp] = (int16_t)w; cse[cp] = loff[w]; cp++;
                            down = true;
                            break;
                        } else if (onst[w] && idx[w] < low[vv]) {
                            low[vv] = idx[w];
                        }
                    }
                    if (down) continue;
                    if (low[vv] == idx[vv]) {
                        int32_t mn = 0x7fffffff, k = sp, sz = 0;
                        do { --k; mn = min(mn, gid[stk[k]]); ++sz; } while (stk[k] != vv);
                        while (sp > k) {
                            int w = stk[--sp];
                            onst[w] = 0;
                            r.label[gid[w]] = mn;
                            r.cls[gid[w]] = CLS_MICE;
                        }
                        atomicAdd((unsigned long long *)(r.hist + sz), 1ull);  // sz <= kLocalV
                        ++nscc;
                    }
                    cp--;
                    if (cp > 0) {
                        int p = csv[cp - 1];
                        if (low[vv] < low[p]) low[p] = low[vv];
                    }
                }
            }
            atomicAdd(r.counters + C_MICE_SCC, (unsigned long long)nscc);
            atomicAdd(r.counters + C_MICE_V, (unsigned long long)nv);
            atomicAdd(r.counters + C_LOCAL_WCC, 1ull);
        }
        __syncthreads();
        // the WCC is done: leave the active map
        for (int i = threadIdx.x; i < nv; i += kLocalThreads) clear_bit(r.A, gid[i]);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Large WCCs: colouring rounds inside classes (the reference's dead
// color_propagation / color_identify, src/color_propagation.h:64-466, made
// the mice stage; it replaces the serial per-pivot mice_fw_bw,
// src/fw_bw.h:1585-1691).
//
// Every active vertex has a priority -- a bijective hash of its id, so
// priorities are random with respect to the graph -- and a class (initially
// its WCC).  Each round a sample of the vertices are pivots: those whose
// priority lies below a threshold that doubles every round (about
// Run::color_pivots -- 1024 by default -- in the first round, every vertex
// after log2(n/1024) rounds), plus
// the residual's minimum-priority vertex.  A pivot's colour starts as its
// priority, every other colour as "none", and colours relax to the minimum
// over the forward ancestors *inside the class*.  A pivot whose colour is its
// own priority is a root; a backward search from all roots at once,
// restricted to the root's colour, collects exactly the root's SCC (every
// ancestor of a member reaches the root, so it has the root's colour).  The
// SCC takes its minimum member id as label and leaves.  Every SCC lies in a
// single colour, so the colour groups of a round (and the vertices no pivot
// reached) are independent sub-problems: a reached vertex's colour becomes
// its class for the next round, an unreached one keeps its class.
//
// Round count and work: with one pivot per class this is forward-backward
// (one SCC per class per round: 108 rounds on the batch workload); with
// every vertex a pivot it is colouring, O(log n) rounds like a treap but each
// vertex's colour drops about ln(#ancestors) times, each drop re-pushing its
// out-edges (10x the work per round).  A sample that grows from small keeps
// the drops per vertex near ln(#pivot ancestors) while classes are large and
// reaches full colouring only once classes are small.
//
// A vertex's class, colour and queued flag share one 64-bit word: class in
// the high half, the 31-bit colour in bits 31..1, and bit 0 set while the
// vertex is NOT in a queue.  An edge check is one load; a relaxation is one
// compare-and-swap that lowers the colour and clears the flag, so the thread
// whose relaxation found the flag set is the one that queues the vertex; a
// pop is one atomicOr that sets the flag and returns the current colour.
// Vertices outside the large WCCs carry the class 0xffffffff, which no live
// class equals (classes are WCC roots and colours, both below 2^31 - 1), so
// the class compare also rejects inactive neighbours.
//
// Both searches run as asynchronous rounds: each CTA takes a slice of the
// global frontier, and its warps work it independently from frontier rings
// in shared memory (a CTA pool passes work to warps that run dry),
// overflowing to the global queue; a grid barrier separates rounds, so
// ring-shaped SCCs cost no grid barrier per hop.
__device__ __forceinline__ uint32_t prio_of(uint32_t v) {
    // bijection on [0, 2^31): xor-shifts and odd multipliers mod 2^31 are
    // invertible there
    v &= 0x7fffffffu;
    v ^= v >> 16;
    v = (v * 0x7feb352du) & 0x7fffffffu;
    v ^= v >> 15;
    v = (v * 0x846ca68bu) & 0x7fffffffu;
    v ^= v >> 16;
    return v;
}
constexpr uint32_t kNoColour = 0x7fffffffu;            // "no pivot reached this vertex"
constexpr unsigned long long kDeadWord = ~0ull;        // class 0xffffffff: outside the large WCCs
__device__ __forceinline__ uint32_t colour_of(unsigned long long w) { return ((uint32_t)w) >> 1; }

constexpr int kCWQ = 256;     // per-warp frontier ring (entries); a power of two
constexpr int kCPool = 1024;  // CTA work pool (entries); a power of two
constexpr int kCLevels = 32;  // default of Run::color_levels: a warp works up to 4 * color_levels chunks of 32 entries per grid round
constexpr int kCPivots = 1024;  // default of Run::color_pivots: pivots of the first colouring round
struct ColorSmem {
    int32_t ring[kWarps][kCWQ];
    int32_t pool[kCPool];
    unsigned long long cursor;  // next unread entry of this CTA's slice of the grid queue
    int phead, ptail;           // pool entries [phead, ptail); guarded by lock
    int active;                 // warps working (not waiting for pool work); guarded by lock
    int lock;
    unsigned long long st[4];   // diagnostics of the round (pops, edges, queued, wait ns); see cst
    long long *cst;             // where they go (null: not recorded)
};

// CTA spin lock in shared memory, taken by one lane.  Holders keep it for a
// few shared-memory operations; the wait is bounded all the same.  Returns
// whether the lock was taken: on a timeout the error word is set and the
// caller skips its critical section (and must not unlock).
__device__ __forceinline__ bool cta_lock(int *l, int *err) {
    for (int i = 0; atomicCAS(l, 0, 1) != 0; ++i) {
        if (i == (1 << 24)) { atomicCAS(err, 0, kErrTimeout); return false; }
        __nanosleep(32);
    }
    __threadfence_block();
    return true;
}
__device__ __forceinline__ void cta_unlock(int *l) {
    __threadfence_block();
    atomicExch(l, 0);
}

// One asynchronous round over the global queue q_in[0..n_in).  KIND 0
// relaxes colours forward inside the class (push the smaller colour to
// out-neighbours of the same class, re-queueing them); KIND 1 grows each
// root's SCC backward inside its colour (claim in-neighbours in F).
//
// Every warp works on its own: it takes 32 entries at a time from its ring
// in shared memory, else from the CTA's slice of the grid queue, else from
// the CTA's pool; it spreads the chunk's edges evenly over its lanes (a warp
// prefix sum over the degrees, each lane finding its edge's owner by a
// binary search over the prefix) and appends the vertices it queues to its
// ring -- or, once its ring holds a chunk and some warp waits for work, to
// the pool (the grid queue when both are full).  No barrier between warps:
// a warp with a long list or slow loads delays no other, and a warp that
// runs dry takes over work another warp generated.  A warp leaves when it
// has worked 4 * color_levels chunks (handing its ring back to the grid
// queue) or when the pool is empty and no warp is working; the CTA then
// hands back the unread rest of its slice and the pool, so no CTA keeps the
// grid barrier waiting; the next grid round spreads that work over all CTAs.
template <typename OffT, int KIND>
__device__ __forceinline__ void color_async_round(const Run<OffT> &r, const Ext<OffT> &x, const int32_t *q_in,
                                                  int64_t n_in, int32_t *q_out, unsigned long long *n_out,
                                                  ColorSmem &sm, long long *cst_arg) {
    unsigned long long *cc = reinterpret_cast<unsigned long long *>(r.qe[0]);  // class | colour | flag
    int32_t *rootof = r.aux2;
    const OffT *beg = KIND == 0 ? r.fw_beg : r.bw_beg;
    const int32_t *adj = KIND == 0 ? r.fw_adj : r.bw_adj;
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    int32_t *ring = sm.ring[threadIdx.x >> 5];
    const int64_t s0 = n_in * blockIdx.x / gridDim.x, s1 = n_in * (blockIdx.x + 1) / gridDim.x;
    __syncthreads();  // the previous round's readers of the shared state are done
    if (threadIdx.x == 0) {
        sm.cursor = (unsigned long long)s0;
        sm.phead = 0;
        sm.ptail = 0;
        sm.active = kWarps;
        sm.lock = 0;
        sm.st[0] = sm.st[1] = sm.st[2] = sm.st[3] = 0ull;
        sm.cst = cst_arg;
    }
    __syncthreads();
    int head = 0, tail = 0;  // ring [head, tail), warp-uniform
    const int cap = 4 * r.color_levels;
    bool capped = false;
    for (int chunk = 0;; ++chunk) {
        if (chunk >= cap) { capped = true; break; }
        int nb = 0;
        int32_t v = -1;
        if (tail != head) {
            nb = min(32, tail - head);
            if (lane < nb) v = ring[(head + lane) & (kCWQ - 1)];
            head += nb;
        } else {
            unsigned long long g = 0;
            if (lane == 0) g = atomicAdd(&sm.cursor, 32ull);
            g = __shfl_sync(kFull, g, 0);
            if ((int64_t)g < s1) {
                nb = (int)min((int64_t)32, s1 - (int64_t)g);
                if (lane < nb) v = __ldcg(q_in + g + lane);
            } else {
                // the pool, waiting for work while another warp may still add some
                int got = 0, pb = 0;
                if (lane == 0) {
                    bool idle = false;
                    const uint64_t t0 = globaltimer();
                    if (sm.cst) atomicAdd(&sm.st[3], 0ull - (unsigned long long)t0);  // diagnostics
                    for (int it = 0;; ++it) {
                        // test without the lock first: waiting warps poll, the lock
                        // stays free for the warps that feed the pool
                        if (!idle || ld_volatile_int(&sm.ptail) != ld_volatile_int(&sm.phead) ||
                            ld_volatile_int(&sm.active) == 0) {
                            if (!cta_lock(&sm.lock, r.err)) break;  // error recorded; this warp stops
                            const int avail = sm.ptail - sm.phead;
                            if (avail > 0) {  // keep the lock until the lanes have read the entries
                                got = min(32, avail);
                                pb = sm.phead;
                                sm.phead += got;
                                if (idle) sm.active += 1;
                                break;
                            }
                            if (!idle) { sm.active -= 1; idle = true; }
                            const bool done = sm.active == 0;
                            cta_unlock(&sm.lock);
                            if (done) break;
                        }
                        if ((it & 63) == 63 && (globaltimer() - t0 > kBarrierTimeoutNs || ld_volatile_int(r.err))) {
                            atomicCAS(r.err, 0, kErrTimeout);
                            break;
                        }
                        __nanosleep(64);
                    }
                    if (sm.cst) atomicAdd(&sm.st[3], (unsigned long long)globaltimer());
                }
                got = __shfl_sync(kFull, got, 0);
                if (got == 0) break;  // nothing left in this CTA for this round
                pb = __shfl_sync(kFull, pb, 0);
                nb = got;
                // the pool entries' vertex state was published before them
                // (block fence on the pushing side); see the push below
                if (lane < nb) v = sm.pool[(pb + lane) & (kCPool - 1)];
                __syncwarp();
                if (lane == 0) cta_unlock(&sm.lock);
            }
        }
        __syncwarp();  // ring slots read above may be refilled below
        // the chunk's vertices: KIND 0 leaves the queue here (sets the flag and
        // reads the colour in one atomic; a lowering after it queues v again,
        // and pushing an older, larger colour meanwhile is harmless)
        unsigned long long pv = 0;
        int32_t rt = 0;
        int64_t deg = 0, base = 0;
        if (lane < nb) {
            pv = KIND == 0 ? atomicOr(cc + v, 1ull) : __ldcg(cc + v);
            if (KIND == 1) rt = __ldcg(rootof + v);
            base = (int64_t)ld_off(beg, v);
            deg = (int64_t)ld_off(beg, v + 1) - base;
        }
        int64_t incl = deg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t t = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += t;
        }
        const int64_t total = __shfl_sync(kFull, incl, 31);
        base -= incl - deg;  // edge index of the chunk's k-th edge, k in this lane's range: base + k
        if (sm.cst && lane == 0) {  // diagnostics, in shared memory (no registers held across the loop)
            atomicAdd(&sm.st[0], (unsigned long long)nb);
            atomicAdd(&sm.st[1], (unsigned long long)total);
        }
        for (int64_t k0 = 0; k0 < total; k0 += 64) {
            int32_t w[2], vo[2];
            unsigned long long po[2], pw[2];
            int32_t ro[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int64_t k = k0 + u * 32 + lane;
                // owner: the number of lanes whose inclusive prefix is <= k
                int o = 0;
#pragma unroll
                for (int st = 16; st; st >>= 1)
                    if (__shfl_sync(kFull, incl, o + st - 1) <= k) o += st;
                const int64_t bo = __shfl_sync(kFull, base, o);
                vo[u] = __shfl_sync(kFull, v, o);
                po[u] = __shfl_sync(kFull, pv, o);
                ro[u] = KIND == 1 ? __shfl_sync(kFull, rt, o) : 0;
                w[u] = k < total ? ld_adj(adj, bo + k) : -1;
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) pw[u] = (w[u] >= 0 && w[u] != vo[u]) ? __ldcg(cc + w[u]) : 0ull;
            // KIND 0: the first compare-and-swap of both sub-batches in flight
            // together (they are independent); a failed one retries alone
            bool pushes[2];
            if (KIND == 0) {
                unsigned long long nw[2], seen[2];
                bool act[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    // the class compare also rejects inactive neighbours (dead
                    // class); lower the colour and clear the flag -- the class
                    // cannot change under a successful swap (it is compared first)
                    const uint32_t cv = colour_of(po[u]);
                    act[u] = w[u] >= 0 && w[u] != vo[u] && (pw[u] >> 32) == (po[u] >> 32) && colour_of(pw[u]) > cv;
                    nw[u] = (po[u] & 0xffffffff00000000ull) | ((unsigned long long)cv << 1);
                }
#pragma unroll
                for (int u = 0; u < 2; ++u) seen[u] = act[u] ? atomicCAS(cc + w[u], pw[u], nw[u]) : pw[u];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    bool lowered = act[u] && seen[u] == pw[u];
                    unsigned long long old = lowered ? pw[u] : seen[u];
                    if (act[u] && !lowered) {
                        const uint32_t cv = colour_of(po[u]);
                        int t = 0;
                        // every failed swap saw a lower colour or a pop's flag
                        for (; t < (1 << 20); ++t) {
                            if ((old >> 32) != (po[u] >> 32) || colour_of(old) <= cv) break;
                            const unsigned long long sn = atomicCAS(cc + w[u], old, nw[u]);
                            if (sn == old) { lowered = true; break; }
                            old = sn;
                        }
                        if (t == (1 << 20)) atomicCAS(r.err, 0, kErrOverflow);
                    }
                    pushes[u] = lowered && (old & 1ull);  // the flag was set: not queued yet
                }
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                bool push;
                if (KIND == 0) {
                    push = pushes[u];
                } else {
                    push = w[u] >= 0 && w[u] != vo[u] && (pw[u] >> 32) == (po[u] >> 32) &&
                           ((pw[u] ^ po[u]) >> 1) == 0 && !bitv(r.F, w[u]) && set_bit(r.F, w[u]);
                    if (push) rootof[w[u]] = ro[u];
                }
                const unsigned m = __ballot_sync(kFull, push);
                if (m) {
                    const int cnt = __popc(m), rank = __popc(m & lt);
                    if (sm.cst && lane == 0) atomicAdd(&sm.st[2], (unsigned long long)cnt);
                    bool placed = false;
                    // one read, broadcast: the branch below must be warp-uniform
                    const int act = __shfl_sync(kFull, ld_volatile_int(&sm.active), 0);
                    if (tail - head >= 32 && act < kWarps) {
                        // share: a warp is waiting for work
                        int pt = -1;
                        if (lane == 0 && cta_lock(&sm.lock, r.err)) {
                            if (kCPool - (sm.ptail - sm.phead) >= cnt) pt = sm.ptail;
                            else cta_unlock(&sm.lock);
                        }
                        pt = __shfl_sync(kFull, pt, 0);
                        if (pt >= 0) {
                            if (push) sm.pool[(pt + rank) & (kCPool - 1)] = w[u];
                            __threadfence_block();  // the vertex's state before the pool entry, for the taking warp
                            __syncwarp();
                            if (lane == 0) {
                                sm.ptail = pt + cnt;
                                cta_unlock(&sm.lock);
                            }
                            placed = true;
                        }
                    }
                    if (!placed && kCWQ - (tail - head) >= cnt) {
                        if (push) ring[(tail + rank) & (kCWQ - 1)] = w[u];
                        tail += cnt;
                        placed = true;
                    }
                    if (!placed) {
                        unsigned long long g = 0;
                        if (lane == 0) g = atomicAdd(n_out, (unsigned long long)cnt);
                        g = __shfl_sync(kFull, g, 0);
                        if (push && VOK((long long)(g + rank), 18)) q_out[g + rank] = w[u];
                    }
                }
            }
        }
        __syncwarp();  // ring appends are visible to the warp's next chunk
    }
    if (capped) {
        if (lane == 0 && cta_lock(&sm.lock, r.err)) {  // no longer working: waiting warps may leave
            sm.active -= 1;
            cta_unlock(&sm.lock);
        }
        if (tail != head) {  // the ring goes back to the grid queue
            const int cnt = tail - head;
            unsigned long long g = 0;
            if (lane == 0) g = atomicAdd(n_out, (unsigned long long)cnt);
            g = __shfl_sync(kFull, g, 0);
            for (int i = lane; i < cnt; i += 32)
                if (VOK((long long)(g + i), 18)) q_out[g + i] = ring[(head + i) & (kCWQ - 1)];
        }
    }
    __syncthreads();
    if (sm.cst && threadIdx.x < 4) atomicAdd((unsigned long long *)sm.cst + threadIdx.x, sm.st[threadIdx.x]);
    // the unread rest of the slice (left by warps that reached their chunk
    // cap) and what is left in the pool go back to the grid queue
    const int64_t from = min((int64_t)sm.cursor, s1), rest = s1 - from;
    const int pn = sm.ptail - sm.phead;
    if (rest + pn > 0) {
        __shared__ unsigned long long s_base;
        if (threadIdx.x == 0) s_base = atomicAdd(n_out, (unsigned long long)(rest + pn));
        __syncthreads();
        const unsigned long long b0 = s_base;
        for (int64_t i = threadIdx.x; i < rest; i += kBlock)
            if (VOK((long long)(b0 + i), 18)) q_out[b0 + i] = __ldcg(q_in + from + i);
        for (int i = threadIdx.x; i < pn; i += kBlock)
            if (VOK((long long)(b0 + rest + i), 18)) q_out[b0 + rest + i] = sm.pool[(sm.phead + i) & (kCPool - 1)];
    }
}

// Asynchronous rounds until the global queue is empty.  Round 0 reads
// (q0, n0); later rounds alternate between the two cascade queues with three
// rotating counters.  Returns the number of rounds, or -1 if a grid barrier
// failed.
template <typename OffT, int KIND>
__device__ __forceinline__ int color_async(const Run<OffT> &r, const Ext<OffT> &x, const int32_t *q0, int64_t n0,
                                           unsigned long long *cqc, ColorSmem &sm, long long *cst = nullptr) {
    for (int lv = 0; lv < (1 << 30); ++lv) {
        const int64_t n = lv == 0 ? n0 : (int64_t)__ldcg(cqc + lv % 3);
        if (n == 0) return lv;
        if (blockIdx.x == 0 && threadIdx.x == 0) cqc[(lv + 2) % 3] = 0ull;
        const int32_t *q = lv == 0 ? q0 : x.cq[lv & 1];
        color_async_round<OffT, KIND>(r, x, q, n, x.cq[(lv + 1) & 1], cqc + (lv + 1) % 3, sm, cst);
        if (!grid_sync(r.gsync, r.err)) return -1;
        if (lv > 64 * (r.V + 2)) {  // colours only decrease; more rounds is a bug
            if (threadIdx.x == 0) atomicCAS(r.err, 0, kErrOverflow);
            return -1;
        }
    }
    return -1;
}

// Runs on the input graph's ids (x.old NULL) unless the compact graph was
// built, or on the compact graph (x.old set, r holding its CSR) if it was;
// the pipeline launches both forms and one of them returns at once.
template <typename OffT>
#ifndef ISPAN_COLOR_MIN_CTAS
#define ISPAN_COLOR_MIN_CTAS 2  // CTAs per SM the colouring kernel is compiled for (registers: 64 at 2)
#endif
__global__ void __launch_bounds__(kBlock, ISPAN_COLOR_MIN_CTAS) k_color(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    __shared__ ColorSmem sm;
    if ((__ldcg(x.ctl + K_CMP_OK) != 0) != (x.old != nullptr)) return;
    const int64_t gt = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    const int64_t nt = (int64_t)gridDim.x * kBlock;
    // class (high half) and colour (low half) of each vertex in one word
    unsigned long long *cc = reinterpret_cast<unsigned long long *>(r.qe[0]);
    const unsigned long long kHi = 0xffffffff00000000ull;
    int32_t *rootof = r.aux2;  // root of the SCC a marked vertex belongs to
    int32_t *mn = r.aux;       // at roots: minimum member id
    int32_t *szc = r.cnt_in;   // at roots: member count (the peel's counters are done)
    unsigned long long *cqc = x.ctl + K_CQ0;
    int cur = 0, rounds = 0;
    int64_t prev_n = INT64_MAX;
    int shift0 = 0;  // first round: pivots are the priorities below 2^(32 - shift0)
    {   // initial classes: the WCCs (parent holds the WCC root until colours overwrite it)
        const int64_t n = (int64_t)__ldcg(x.ctl + K_LARGE);
        while (shift0 < 30 && (n >> (shift0 + 1)) >= r.color_pivots) ++shift0;
        if (blockIdx.x == 0 && threadIdx.x == 0) x.ctl[K_MINPRIO0] = ~0ull;
        if (n == 0) return;
        // every word dead first: neighbours outside the large WCCs fail the class
        // compare (the compact graph has no such neighbours; its ids are < n)
        const int64_t nw = x.old ? n : r.V;
        for (int64_t i = gt; i < nw; i += nt) cc[i] = kDeadWord;
        if (!grid_sync(r.gsync, r.err)) return;
        uint32_t pm = 0xffffffffu;
        for (int64_t i = gt; i < n; i += nt) {
            int32_t v = x.large[0][i];
            cc[v] = ((unsigned long long)(uint32_t)r.parent[orig_id(x, v)] << 32) |
                    ((unsigned long long)kNoColour << 1) | 1ull;
            pm = min(pm, prio_of((uint32_t)v));
        }
        pm = __reduce_min_sync(0xffffffffu, pm);
        if ((threadIdx.x & 31) == 0) atomicMin(x.ctl + K_MINPRIO0, (unsigned long long)pm);
        if (!grid_sync(r.gsync, r.err)) return;
    }
    for (int guard = 0; guard < (1 << 30); ++guard) {
        const int64_t n = (int64_t)__ldcg(x.ctl + (cur == 0 ? K_LARGE : K_LARGE2));
        if (n == 0) break;
        if (n >= prev_n) {  // every round labels the SCC of each class's lowest priority
            if (threadIdx.x == 0) atomicCAS(r.err, 0, kErrOverflow);
            return;
        }
        prev_n = n;
        ++rounds;
        const int32_t *L = x.large[cur];
        // pivots: priority below the round's threshold, or the residual's minimum
        const int shift = max(0, shift0 - (rounds - 1));
        const unsigned long long thr = 1ull << (31 - shift);
        const unsigned long long minp = __ldcg(x.ctl + K_MINPRIO0 + cur);
        unsigned long long *next_minp = x.ctl + K_MINPRIO0 + (cur ^ 1);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            cqc[0] = 0; cqc[1] = 0; cqc[2] = 0;
            x.ctl[cur == 0 ? K_LARGE2 : K_LARGE] = 0;
        }
        if (!grid_sync(r.gsync, r.err)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) *next_minp = ~0ull;  // read above, before the barrier
        for (int64_t i = gt; i - threadIdx.x < n; i += nt) {
            bool piv = false;
            int32_t v = 0;
            if (i < n) {
                v = L[i];
                const uint32_t p = prio_of((uint32_t)v);
                piv = p < thr || p <= minp;
                // a pivot starts queued (flag clear) with its priority as colour
                cc[v] = (__ldcg(cc + v) & kHi) | (piv ? (unsigned long long)p << 1 : ((unsigned long long)kNoColour << 1) | 1ull);
                clear_bit(r.F, v);  // F: SCC mark of this round
            }
            wl_append(piv, v, x.cq[0], cqc + 0);
        }
        if (!grid_sync(r.gsync, r.err)) return;
        // forward min-colour relaxation from the pivots; cqc[0] is freed by
        // color_async only after every CTA has read it here
        const int64_t npiv = (int64_t)__ldcg(cqc + 0);
        // diagnostics on request (exact statistics): pops, edges, pushes and
        // pool-wait time of the forward relaxation, summed over warps
        long long *cst = (r.flags & ISPAN_F_EXACT_STATS) && rounds <= kTraceLevels
                             ? r.trace + ((long long)3 * kTraceLevels + rounds - 1) * 4
                             : nullptr;
        const int fw_rounds = color_async<OffT, 0>(r, x, x.cq[0], npiv, cqc, sm, cst);
        if (fw_rounds < 0) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) { cqc[0] = 0; cqc[1] = 0; cqc[2] = 0; }
        if (!grid_sync(r.gsync, r.err)) return;
        for (int64_t i = gt; i - threadIdx.x < n; i += nt) {  // roots
            bool rt = false;
            int32_t v = 0;
            if (i < n) {
                v = L[i];
                const uint32_t p = prio_of((uint32_t)v);
                // colours are pivot priorities, so a match means v is a pivot
                // unless v's priority is the "none" value itself
                rt = colour_of(__ldcg(cc + v)) == p && (p < thr || p <= minp);
                if (rt) {
                    set_bit(r.F, v);
                    rootof[v] = v;
                    mn[v] = orig_id(x, v);
                    szc[v] = 0;
                }
            }
            wl_append(rt, v, x.cq[0], cqc + 0);
        }
        if (!grid_sync(r.gsync, r.err)) return;
        // the roots' count stays in cqc[0] until color_async frees that slot
        // two rounds later, long after every CTA has read it here
        const int bw_rounds = color_async<OffT, 1>(r, x, x.cq[0], (int64_t)__ldcg(cqc + 0), cqc, sm);
        if (bw_rounds < 0) return;
        if (blockIdx.x == 0 && threadIdx.x == 0 && rounds <= kTraceLevels) {  // diagnostics
            long long *t = r.trace + ((long long)2 * kTraceLevels + rounds - 1) * 4;
            t[0] = rounds | ((long long)fw_rounds << 16) | ((long long)bw_rounds << 40);
            t[1] = n;
            t[2] = npiv;
            t[3] = (long long)globaltimer();
        }
        // a marked vertex's root is a vertex id (compact ids are smaller
        // still); anything else is an internal error, recorded, and the
        // access skipped (the root tables hold V entries)
        const int64_t idb = r.V;
        for (int64_t i = gt; i < n; i += nt) {  // minimum member id and size per SCC
            int32_t v = L[i];
            if (bitv(r.F, v)) {
                const int32_t rv = __ldcg(rootof + v);
                if ((uint64_t)(int64_t)rv >= (uint64_t)idb) {
                    atomicCAS(r.err, 0, kErrOverflow);
                    continue;
                }
                atomicMin(mn + rv, orig_id(x, v));  // labels are original ids
                atomicAdd(szc + rv, 1);
            }
        }
        if (!grid_sync(r.gsync, r.err)) return;
        int64_t nl = 0, nroots = 0;
        uint32_t pm = 0xffffffffu;
        for (int64_t i = gt; i - threadIdx.x < n; i += nt) {  // labels, sizes; the rest continues
            bool keep = false;
            int32_t v = 0;
            if (i < n) {
                v = L[i];
                if (bitv(r.F, v)) {
                    int32_t rv = __ldcg(rootof + v);
                    if ((uint64_t)(int64_t)rv >= (uint64_t)idb) rv = v;  // recorded above as an error
                    const int32_t ov = orig_id(x, v);
                    r.label[ov] = __ldcg(mn + rv);
                    r.cls[ov] = CLS_MICE;
                    clear_bit(r.A, ov);
                    cc[v] = kDeadWord;
                    ++nl;
                    if (rv == v) {  // one histogram entry per SCC, at its root
                        const int32_t sz = __ldcg(szc + v);
                        if (sz < kHistCap) {
                            atomicAdd((unsigned long long *)(r.hist + sz), 1ull);
                        } else {
                            unsigned long long k = atomicAdd(r.counters + C_BIG, 1ull);
                            if (k < kBigCap) r.hist[kHistCap + k] = sz;
                        }
                        ++nroots;
                    }
                } else {
                    keep = true;
                    const unsigned long long pv = __ldcg(cc + v);
                    const uint32_t c = colour_of(pv);
                    // reached: its colour is its next class; unreached: it keeps its class
                    cc[v] = (c != kNoColour ? ((unsigned long long)c << 32) : (pv & kHi)) |
                            ((unsigned long long)kNoColour << 1) | 1ull;
                    pm = min(pm, prio_of((uint32_t)v));
                }
            }
            wl_append(keep, v, x.large[cur ^ 1], x.ctl + (cur == 0 ? K_LARGE2 : K_LARGE));
        }
        pm = __reduce_min_sync(0xffffffffu, pm);
        if ((threadIdx.x & 31) == 0 && pm != 0xffffffffu) atomicMin(next_minp, (unsigned long long)pm);
        int64_t a = block_sum64(nl, sh), b = block_sum64(nroots, sh);
        if (threadIdx.x == 0) {
            if (a) atomicAdd(r.counters + C_MICE_V, (unsigned long long)a);
            if (b) atomicAdd(r.counters + C_MICE_SCC, (unsigned long long)b);
        }
        if (!grid_sync(r.gsync, r.err)) return;
        cur ^= 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) r.counters[C_COLOR_ROUNDS] = (unsigned long long)rounds;
}

// ---------------------------------------------------------------------------
// Final labels of the giant SCCs, histogram entries of the classes whose
// sizes are fixed, and the per-graph giant sizes.  Any vertex still active
// here is an internal error.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_finalize(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    constexpr int U = 4;
    const int lane = lane_id();
    const int64_t gw = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int64_t nw = (int64_t)gridDim.x * kWarps;
    for (int64_t wb = gw * U; wb < r.W; wb += nw * U) {
        uint32_t t[U], b[U], a[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            const int64_t wi = wb + j;
            t[j] = wi < r.W ? r.T[wi] : 0u;
            b[j] = wi < r.W ? r.B[wi] : 0u;
            a[j] = wi < r.W ? r.A[wi] : 0u;
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
            if (a[j] && lane == 0) atomicCAS(r.err, 0, kErrOverflow);  // every vertex must be labelled
            const int64_t v = (wb + j) * 32 + lane;
            int32_t gm = 0;
            if (b[j]) {  // one graph per word unless it straddles a boundary
                if (r.nseg == 1) {
                    gm = r.gmin[0];
                } else {
                    int s0 = 0, s1 = 0;
                    if (lane == 0) {
                        s0 = seg_of(r.vbase, r.nseg, (wb + j) * 32);
                        s1 = seg_of(r.vbase, r.nseg, min((wb + j) * 32 + 31, r.V - 1));
                    }
                    s0 = __shfl_sync(kFull, s0, 0);
                    s1 = __shfl_sync(kFull, s1, 0);
                    gm = r.gmin[s0 == s1 ? s0 : seg_of(r.vbase, r.nseg, v)];
                }
            }
            if ((b[j] >> lane) & 1u) r.label[v] = gm;
            else if ((t[j] >> lane) & 1u) r.label[v] = (int32_t)v;
        }
    }
    const int64_t gt = (int64_t)blockIdx.x * kBlock + threadIdx.x;
    for (int64_t sg = gt; sg < r.nseg; sg += (int64_t)gridDim.x * kBlock) {
        unsigned long long sz = r.gsize[sg];
        if (!sz) continue;
        atomicAdd(r.counters + C_GIANTS, 1ull);
        if (sz < (unsigned long long)kHistCap) {
            atomicAdd((unsigned long long *)(r.hist + sz), 1ull);
        } else {
            unsigned long long k = atomicAdd(r.counters + C_BIG, 1ull);
            if (k < kBigCap) r.hist[kHistCap + k] = (int64_t)sz;
        }
    }
    if (gt == 0) {
        unsigned long long t1 = r.counters[C_TRIM1], t2 = r.counters[C_TRIM2], t3 = r.counters[C_TRIM3];
        atomicAdd((unsigned long long *)(r.hist + 1), t1);
        atomicAdd((unsigned long long *)(r.hist + 2), t2 / 2);
        atomicAdd((unsigned long long *)(r.hist + 3), t3 / 3);
    }
}

}  // namespace ispan

// bfs.cuh -- direction-optimising reachability for the giant ("elephant")
// SCC.  Replaces fw_bfs_fq_queue (src/fw_bw.h:396-698) and bw_bfs_fq_queue
// (src/fw_bw.h:944-1248) of the reference.
//
// One persistent, cooperatively launched kernel runs every level of one
// search; levels are separated by a bounded grid barrier and the level/mode
// control is computed on the device, identically in every CTA, from the
// level's counters -- no host round trip per level.
//
// Modes (the reference's three, re-designed for the GPU):
//   TD   top-down over a frontier queue.  The queue is an edge prefix built by
//        the producers (see q_append), so work is split into equal chunks of
//        kChunk edges regardless of the degree skew: a hub's adjacency is
//        spread over many CTAs, a run of low-degree vertices shares one chunk
//        (this edge-balanced split replaces binning vertices by degree into
//        thread/warp/CTA expansion).  Each thread reads four consecutive
//        adjacency entries, as one int4 load when they are 16-byte aligned in
//        one list.
//   BU   bottom-up pull over the 1-bit maps, one warp per 32-vertex word.
//        Each unvisited candidate scans its reverse edges and stops at the
//        first visited neighbour of any level (the reference's "Rsync" rule),
//        first alone for up to kBuLane edges, then with its warp.
//   TAIL top-down with CTA 0 alone while the frontier is small, levels
//        separated by __syncthreads only, so long thin tails do not pay one
//        grid barrier per level (the reference's per-thread async ring queue).
// Switching follows the reference's rules with edge counts in place of
// vertex_count * avg_degree: TD -> BU when frontier edges > unexplored
// edges / alpha; BU -> TD when the frontier < |candidates| / beta or the level
// exceeds gamma; TD <-> TAIL on the frontier size.
//
// DIR 0 (forward):  visit map F, restricted to A, expands out-edges.
// DIR 1 (backward): visit map B, restricted to F, expands in-edges -- or,
// when both searches run at the same time (kRunPair; small graphs, whose
// levels are latency-bound), restricted to A, in its own queues, with its
// own grid barrier and the map D for its bottom-up snapshots.  The pivot SCC
// is F & B either way.
#pragma once
#include "common.cuh"

namespace ispan {

constexpr int kBuLane = 16;          // edges a lane scans alone in bottom-up
constexpr int kLQ = 2048;               // per-CTA local frontier (shared memory) in the async mode
constexpr int kAsyncDeg = 16;           // default of Run::async_deg: vertices up to this degree are expanded locally
constexpr int kAsyncMaxLevels = 4096;   // local levels before a CTA hands its frontier back
constexpr int64_t kAsyncV = 65536;      // defaults of Run::async_v: frontier size that enters the async mode ...
constexpr int64_t kAsyncE = 262144;     // ... and Run::async_e: frontier edges
constexpr int64_t kPairMaxV = 1 << 20;  // graphs up to this many vertices run their two searches at once

enum BfsMode : int { M_TD = 0, M_BU = 1, M_ASYNC = 2, M_DONE = 3 };

// level stats slot (4 x u64 per slot, 3 slots): newly visited, their
// expansion-side degree sum, their other-side degree sum, spare
struct LvlSlot { unsigned long long nvis, m_next, m_other, spare; };

// shared control written by CTA 0 after a tail phase, read by all after the
// barrier: level, mode, queue parity
struct BfsCtl { int level, mode, done, pad; };

template <typename OffT, int DIR>
struct BfsDir {
    // expansion side (TD follows these edges), pull side (BU scans these)
    const OffT *xbeg, *pbeg, *obeg;
    const int32_t *xadj, *padj;
    const uint32_t *R;   // restriction map (A or F)
    uint32_t *Vm;        // visit map (F or B)
    __device__ BfsDir(const Run<OffT> &r) {
        if (DIR == 0) {
            xbeg = r.fw_beg; xadj = r.fw_adj; pbeg = r.bw_beg; padj = r.bw_adj; obeg = r.bw_beg;
            R = r.A; Vm = r.F;
        } else {
            xbeg = r.bw_beg; xadj = r.bw_adj; pbeg = r.fw_beg; padj = r.fw_adj; obeg = r.fw_beg;
            R = (r.flags & kRunPair) ? r.A : r.F;
            Vm = r.B;
        }
    }
    __device__ __forceinline__ int64_t xdeg(int64_t v) const { return ld_off(xbeg, v + 1) - ld_off(xbeg, v); }
    __device__ __forceinline__ int64_t odeg(int64_t v) const { return ld_off(obeg, v + 1) - ld_off(obeg, v); }
};

// Shared staging of one chunk's queue slots (at most kChunk + 1 of them, as
// every queued vertex has at least one edge).
struct TdSmem {
    int64_t qe[kChunk + 1];    // edge prefix of each slot
    int64_t base[kChunk + 1];  // adjacency start of the slot's vertex minus its prefix
    int wn[kWarps];            // per-warp item counts and degree sums for the
    int64_t wd[kWarps];        // CTA-level reservation
    unsigned long long base_pk;
};

// CTA-level reservation of queue slots and edge ranges: one 64-bit atomic per
// CTA and chunk (a per-warp atomic on the single queue counter serialises at
// L2 when a level expands hundreds of millions of edges).  All threads call it.
template <typename Sm>
__device__ __forceinline__ void q_reserve_block(int n, int64_t dsum, unsigned long long *pk, int64_t &slot0,
                                                int64_t &eb0, Sm &sm) {
    const int lane = lane_id(), warp = threadIdx.x >> 5;
    int ni = n;
    int64_t di = dsum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int yn = __shfl_up_sync(kFull, ni, o);
        int64_t yd = __shfl_up_sync(kFull, di, o);
        if (lane >= o) { ni += yn; di += yd; }
    }
    if (lane == 31) { sm.wn[warp] = ni; sm.wd[warp] = di; }
    __syncthreads();
    if (threadIdx.x == 0) {
        int tn = 0;
        int64_t td = 0;
        for (int i = 0; i < kWarps; ++i) {
            int cn = sm.wn[i];
            int64_t cd = sm.wd[i];
            sm.wn[i] = tn;
            sm.wd[i] = td;
            tn += cn;
            td += cd;
        }
        sm.base_pk = tn ? atomicAdd(pk, ((unsigned long long)td << kCountBits) | (unsigned long long)tn) : 0ull;
    }
    __syncthreads();
    unsigned long long base = sm.base_pk;
    slot0 = (int64_t)(base & kCountMask) + sm.wn[warp] + (ni - n);
    eb0 = (int64_t)(base >> kCountBits) + sm.wd[warp] + (di - dsum);
}

// Expand one chunk of the current queue (top-down), kPer consecutive virtual
// edges per thread.  All threads of the CTA call it.  The chunk's slots are
// first staged into shared memory in one parallel round (prefix and
// adjacency base of each slot), so mapping an edge to its adjacency position
// is a shared-memory search, not a chain of dependent global loads.  The
// thread's targets, their status bits, the claims and the degrees are then
// each loaded as one independent batch, and the new vertices are appended
// with one atomic per warp.
template <typename OffT, int DIR>
__device__ __forceinline__ void td_chunk(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int64_t c,
                                         int64_t nchunks, int64_t qcount, int64_t qedges, int cur,
                                         unsigned long long *pk_next, int64_t &nvis, int64_t &msum_next,
                                         int64_t &msum_other, int tid, TdSmem &sm) {
    const int32_t *qv = r.qv[cur];
    const int64_t *qe = r.qe[cur];
    const int32_t *qc = r.qchunk[cur];
    int nx = cur ^ 1;
    int64_t e0 = c * kChunk;
    int64_t e1 = min(e0 + (int64_t)kChunk, qedges);
    int64_t s_lo = __ldcg(qc + c);
    int64_t s_hi = (c + 1 < nchunks) ? (int64_t)__ldcg(qc + c + 1) : qcount - 1;
    bool ok = ICHK(s_lo >= 0 && s_lo <= s_hi && s_hi < qcount && s_hi - s_lo <= kChunk, 20,
                   (s_lo << 32) | (s_hi & 0xffffffff));
    const int ns = ok ? (int)(s_hi - s_lo + 1) : 0;
    __syncthreads();  // the previous chunk's readers are done with the staging
    for (int i = tid; i < ns; i += kBlock) {
        int64_t q = __ldcg(qe + s_lo + i);
        int32_t v = __ldcg(qv + s_lo + i);
        sm.qe[i] = q;
        sm.base[i] = ld_off(d.xbeg, v) - q;
    }
    __syncthreads();
    constexpr int kPer = kChunk / kBlock;
    const int64_t my0 = e0 + (int64_t)tid * kPer;
    int32_t w[kPer];
    if (ns > 0 && my0 < e1) {
        int lo = 0, hi = ns - 1;
        while (lo < hi) {  // last staged slot with prefix <= my0
            int mid = (lo + hi + 1) >> 1;
            if (sm.qe[mid] <= my0) lo = mid; else hi = mid - 1;
        }
        int i = lo;
        // the thread's four virtual edges in one adjacency list at a 16-byte
        // aligned address: one vectorised int4 load; otherwise (a list
        // boundary inside the group, the chunk's end, a misaligned address)
        // one load per edge
        const int64_t p0 = sm.base[i] + my0;
        const bool one_list = my0 + kPer <= e1 && (i + 1 >= ns || sm.qe[i + 1] >= my0 + kPer);
#ifdef ISPAN_CHECKED
        const bool vec = false;  // the checked build range-checks every id
        (void)one_list;
#else
        const bool vec = kPer == 4 && one_list && ((uintptr_t)(d.xadj + p0) & 15) == 0;
#endif
        if (vec) {
            const int4 q = __ldg(reinterpret_cast<const int4 *>(d.xadj + p0));
            w[0] = q.x; w[1] = q.y; w[2] = q.z; w[3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < kPer; ++k) {
                int64_t e = my0 + k;
                w[k] = -1;
                if (e < e1) {
                    while (i + 1 < ns && sm.qe[i + 1] <= e) ++i;
                    w[k] = ld_adj(d.xadj, sm.base[i] + e);
                }
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < kPer; ++k) w[k] = -1;
    }
    bool cand[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        bool inr = w[k] >= 0 && bit(d.R, w[k]);
        bool seen = w[k] >= 0 && bitv(d.Vm, w[k]);
        cand[k] = inr && !seen;
    }
#pragma unroll
    for (int k = 0; k < kPer; ++k)
        if (!(cand[k] && set_bit(d.Vm, w[k]))) w[k] = -1;
    int n = 0;
    int64_t dsum = 0;
    int32_t dg[kPer];  // a single vertex's degree fits int32
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        dg[k] = 0;
        if (w[k] >= 0) {
            dg[k] = (int32_t)d.xdeg(w[k]);
            nvis += 1;
            if (dg[k] > 0) { ++n; dsum += dg[k]; } else { w[k] = -1; }  // nothing to expand
        }
    }
    msum_next += dsum;
    int64_t slot, eb;
    q_reserve_block(n, dsum, pk_next, slot, eb, sm);
    int32_t *qvn = r.qv[nx];
    int64_t *qen = r.qe[nx];
    int32_t *qcn = r.qchunk[nx];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (w[k] < 0) continue;
        if (ICHK(slot < r.V, 10, slot)) {
            qvn[slot] = w[k];
            qen[slot] = eb;
            int64_t c0 = (eb + kChunk - 1) / kChunk, c1 = (eb + dg[k] - 1) / kChunk;
            for (int64_t cc = c0; cc <= c1; ++cc)
                if (ICHK(cc >= 0 && cc < g_qcap_or(cc + 1), 11, cc)) qcn[cc] = (int32_t)slot;
        }
        ++slot;
        eb += dg[k];
    }
}

// Bottom-up pull of one candidate per lane (v < 0: no candidate).  A lane
// scans its candidate's reverse edges in batches of 4 (edge loads, then bit
// loads, each batch in flight together) for up to kBuLane edges; longer lists
// are finished by the whole warp, 32 edges per step.  Returns found.
template <typename OffT, int DIR>
__device__ __forceinline__ bool bu_pull(const BfsDir<OffT, DIR> &d, int64_t v, int64_t &pdeg) {
    const int lane = lane_id();
    bool found = false;
    int64_t e = 0, end = 0;
    pdeg = 0;
    if (v >= 0) {
        e = ld_off(d.pbeg, v);
        end = ld_off(d.pbeg, v + 1);
        pdeg = end - e;
        const int64_t cap = min(end, e + (int64_t)kBuLane);
        while (e < cap && !found) {
            int32_t u[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) u[q] = (e + q < cap) ? ld_adj(d.padj, e + q) : -1;
            bool h = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) h |= u[q] >= 0 && bitv(d.Vm, u[q]);
            found = h;
            e = min(e + 4, cap);
        }
    }
    unsigned rm = __ballot_sync(kFull, v >= 0 && !found && e < end);
    while (rm) {  // the warp finishes long scans one lane at a time
        int l = __ffs(rm) - 1;
        rm &= rm - 1;
        int64_t le = __shfl_sync(kFull, e, l), lend = __shfl_sync(kFull, end, l);
        bool hit = false;
        // 128 edges per step: four ids per lane, then their four visit bits,
        // each group of loads in flight together (a hub's list costs a
        // quarter of the dependent round trips of 32-edge steps)
        for (int64_t b = le; b < lend; b += 128) {
            int32_t u[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int64_t i = b + q * 32 + lane;
                u[q] = i < lend ? ld_adj(d.padj, i) : -1;
            }
            bool h = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) h |= u[q] >= 0 && bitv(d.Vm, u[q]);
            if (__any_sync(kFull, h)) { hit = true; break; }
        }
        if (lane == l) found = hit;
    }
    return found;
}

// Bottom-up over the bitmap.  Each warp loads 32 words at once (one
// coalesced load per map) and records the snapshot; the candidates of those
// words are then dealt out one per lane (n-th set bit selection), so dense
// and sparse levels both keep every lane busy.  Found bits are combined per
// word before the atomic OR.  Warps take their 32-word groups from a level
// counter, so a warp held up by long reverse lists takes fewer groups
// instead of holding back the grid barrier.
template <typename OffT, int DIR>
__device__ __forceinline__ void bu_words(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int64_t gwarp,
                                         int64_t nwarps, unsigned long long *next_group, int64_t &nvis,
                                         int64_t &msum_next, int64_t &msum_other) {
    const int lane = lane_id();
    // words per group: 32 (one per lane) when there are groups enough for
    // every warp, fewer on small graphs so that more warps get candidates
    int gsz = 32;
    while (gsz > 1 && (int64_t)(r.W + gsz - 1) / gsz < nwarps) gsz >>= 1;
    // the first group is the warp's own index (no atomic; on small graphs
    // most warps have none), later ones come from the counter
    for (int64_t g = gwarp;;) {
        const int64_t wb = g * gsz;
        if (wb >= r.W) break;
        const int64_t my = wb + lane;
        const bool mine = lane < gsz && my < r.W;
        uint32_t vis = mine ? __ldcg(d.Vm + my) : 0u;
        uint32_t cnd = mine ? (__ldg(d.R + my) & ~vis) : 0u;
        if (mine) r.P[my] = vis;  // snapshot for a later switch to top-down
        int c = __popc(cnd), incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(kFull, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl = incl - c;
        const int total = __shfl_sync(kFull, incl, 31);
        for (int base = 0; base < total; base += 32) {
            const int t = base + lane;
            int j = 0;  // lane (word) whose candidate range holds t
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                int ex = __shfl_sync(kFull, excl, (j + step) & 31);
                if (j + step < 32 && ex <= t) j += step;
            }
            uint32_t mj = __shfl_sync(kFull, cnd, j);
            int kth = t - __shfl_sync(kFull, excl, j);
            int64_t v = -1;
            if (t < total) v = (wb + j) * 32 + (int)__fns(mj, 0, kth + 1);
            int64_t pdeg;
            bool found = bu_pull<OffT, DIR>(d, v, pdeg);
            // combine the found bits of lanes that share a word
            int64_t word = found ? (v >> 5) : -1 - lane;
            unsigned grp = __match_any_sync(kFull, word);
            uint32_t mybit = found ? (1u << (v & 31)) : 0u;
            uint32_t orv = __reduce_or_sync(grp, mybit);
            if (found && lane == __ffs(grp) - 1) atomicOr(d.Vm + word, orv);
            if (found) {  // expansion-side degrees are not needed once a search is bottom-up
                nvis += 1;
                msum_other += pdeg;
            }
        }
        // more groups than warps: the next one comes from the level counter
        // (on small graphs every warp's own group is the only one, and 10^3
        // warps' atomics on one counter would cost more than the level)
        if ((r.W + gsz - 1) / gsz <= nwarps) break;
        unsigned long long nx = 0;
        if (lane == 0) nx = atomicAdd(next_group, 1ull);
        g = nwarps + (int64_t)__shfl_sync(kFull, nx, 0);
    }
    (void)msum_next;
}

// Single-vertex append to the global frontier queue (any thread, no warp
// uniformity needed): reserve one slot and its edge range, then write.
__device__ __forceinline__ void q_append_one(int32_t v, int64_t deg, int32_t *qv, int64_t *qe, int32_t *qchunk,
                                             unsigned long long *pk, int64_t cap_v) {
    unsigned long long base = atomicAdd(pk, ((unsigned long long)deg << kCountBits) | 1ull);
    int64_t slot = (int64_t)(base & kCountMask), eb = (int64_t)(base >> kCountBits);
    if (ICHK(slot < cap_v, 10, slot)) {
        qv[slot] = v;
        qe[slot] = eb;
        int64_t c0 = (eb + kChunk - 1) / kChunk, c1 = (eb + deg - 1) / kChunk;
        for (int64_t c = c0; c <= c1; ++c)
            if (ICHK(c >= 0 && c < g_qcap_or(c + 1), 11, c)) qchunk[c] = (int32_t)slot;
    }
}

struct AsyncSmem {
    int32_t lq[2][kLQ];
    int cnt[2];
    int flush;  // hand the local frontier back to the grid at the next level
};

constexpr int kAsyncFlush = kLQ / 2;  // a CTA's local frontier above this is work for the whole grid

// Asynchronous top-down round (the GPU form of the reference's per-thread
// ring-buffer mode, src/fw_bw.h:506-544).  Each CTA takes a slice of the
// current frontier and runs its own BFS on it to exhaustion: the local
// frontier lives in shared memory and local levels are separated by
// __syncthreads only, so a long thin tail costs no grid barrier per level.
// Vertices claimed here with more than kAsyncDeg edges, and local overflow,
// go to the global next queue (expanded edge-balanced in the next round).
// Claims use the same atomic visit map, so any interleaving is a valid
// search: the reached set does not depend on the order.
template <typename OffT, int DIR>
__device__ __forceinline__ void async_round(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int cur, int64_t qcount,
                                            unsigned long long *pk_next, int64_t &nvis, int64_t &msum_next,
                                            int64_t &msum_other, AsyncSmem &sm) {
    const int tid = threadIdx.x;
    const int nx = cur ^ 1;
    const int32_t *qv = r.qv[cur];
    int32_t *qvn = r.qv[nx];
    int64_t *qen = r.qe[nx];
    int32_t *qcn = r.qchunk[nx];
    const int64_t s0 = qcount * blockIdx.x / gridDim.x, s1 = qcount * (blockIdx.x + 1) / gridDim.x;
    for (int64_t bs = s0; bs < s1; bs += kLQ) {
        const int n0 = (int)min((int64_t)kLQ, s1 - bs);
        __syncthreads();
        for (int i = tid; i < n0; i += kBlock) sm.lq[0][i] = __ldcg(qv + bs + i);
        if (tid == 0) { sm.cnt[0] = n0; sm.cnt[1] = 0; sm.flush = 0; }
        __syncthreads();
        int c = 0;
        for (int it = 0; it < kAsyncMaxLevels; ++it) {
            const int n = sm.cnt[c];
            if (n == 0) break;
            // a frontier that widened (here, or grid-wide in the global queue)
            // goes back to the edge-balanced top-down kernel
            const bool last = it == kAsyncMaxLevels - 1 || sm.flush;
            for (int i = tid; i < n; i += kBlock) {
                const int32_t v = sm.lq[c][i];
                const int64_t x0 = ld_off(d.xbeg, v), x1 = ld_off(d.xbeg, v + 1);
                // vertices handed in from the global queue (it == 0) are always
                // expanded here, whatever their degree, so every round makes
                // progress; locally found ones are at most kAsyncDeg
                if (last) {  // level cap: the rest is expanded edge-balanced next round
                    q_append_one(v, x1 - x0, qvn, qen, qcn, pk_next, r.V);
                    msum_next += x1 - x0;
                    continue;
                }
                for (int64_t e = x0; e < x1; e += 4) {
                    int32_t w[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) w[q] = e + q < x1 ? ld_adj(d.xadj, e + q) : -1;
                    bool cand[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        bool inr = w[q] >= 0 && bit(d.R, w[q]);
                        bool seen = w[q] >= 0 && bitv(d.Vm, w[q]);
                        cand[q] = inr && !seen;
                    }
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (!(cand[q] && set_bit(d.Vm, w[q]))) continue;
                        int64_t dg = d.xdeg(w[q]);
                        nvis += 1;
                        if (dg == 0) continue;
                        int pos = dg <= r.async_deg ? atomicAdd(&sm.cnt[c ^ 1], 1) : kLQ;
                        if (pos < kLQ) {
                            sm.lq[c ^ 1][pos] = w[q];
                        } else {  // a hub, or the local frontier is full
                            q_append_one(w[q], dg, qvn, qen, qcn, pk_next, r.V);
                            msum_next += dg;
                        }
                    }
                }
            }
            __syncthreads();
            if (tid == 0) {
                sm.cnt[c ^ 1] = min(sm.cnt[c ^ 1], kLQ);  // claims beyond the capacity went global
                sm.cnt[c] = 0;
                const int64_t global_q = (int64_t)(__ldcg(pk_next) & kCountMask);
                sm.flush = sm.cnt[c ^ 1] > kAsyncFlush || global_q > r.async_v;
            }
            __syncthreads();
            if (last) break;  // this level only handed vertices on
            c ^= 1;
        }
    }
}

// Rebuild the top-down queue from the vertices visited during the last
// bottom-up level (visit map minus its snapshot).
template <typename OffT, int DIR>
__device__ __forceinline__ void rebuild_queue(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int nx,
                                              unsigned long long *pk, int64_t w_begin, int64_t w_stride) {
    const int lane = lane_id();
    for (int64_t wb = w_begin * 32; wb < r.W; wb += w_stride * 32) {
        const int64_t my = wb + lane;
        uint32_t nw = my < r.W ? (__ldcg(d.Vm + my) & ~__ldcg(r.P + my)) : 0u;
        unsigned has = __ballot_sync(kFull, nw != 0);
        while (has) {
            int l = __ffs(has) - 1;
            has &= has - 1;
            uint32_t m = __shfl_sync(kFull, nw, l);
            bool me = (m >> lane) & 1u;
            int64_t v = (wb + l) * 32 + lane;
            int64_t dg = me ? d.xdeg(v) : 0;
            q_append(me, (int32_t)v, dg, r.qv[nx], r.qe[nx], r.qchunk[nx], pk, r.V);
        }
    }
}

template <typename OffT, int DIR>
__global__ void __launch_bounds__(kBlock, 2) k_bfs(Run<OffT> r, BfsCtl *ctl) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    constexpr size_t kSm = sizeof(TdSmem) > sizeof(AsyncSmem) ? sizeof(TdSmem) : sizeof(AsyncSmem);
    __shared__ __align__(16) unsigned char smraw[kSm];
    TdSmem &tdsm = *reinterpret_cast<TdSmem *>(smraw);
    AsyncSmem &asm_ = *reinterpret_cast<AsyncSmem *>(smraw);
    const BfsDir<OffT, DIR> d(r);
    const int tid = threadIdx.x;
    const int64_t gwarp = ((int64_t)blockIdx.x * kBlock + tid) >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * kWarps;
    LvlSlot *slots = reinterpret_cast<LvlSlot *>(r.lvl);
    (void)ctl;

    // budget for the alpha rule: unexplored expansion-side edges.  The
    // backward search takes the in-degree sum over the active set, an upper
    // bound of the sum over F (the forward search does not sum its reached
    // vertices' in-degrees: two more random offset loads per vertex);
    // a backward search running beside the forward one also counts its
    // candidates over A
    const bool over_a = DIR == 0 || (r.flags & kRunPair);
    int64_t m_unexpl = (int64_t)(DIR == 0 ? r.counters[C_MU0] : r.counters[C_MU0_IN]);
    const int64_t n_total = (int64_t)(over_a ? r.counters[C_ACTIVE0] : r.counters[C_FW_SIZE]);
    int level = 0, mode = M_TD;
    bool left_bu = false;  // like the reference, a search never returns to bottom-up
    int64_t total_vis = 0;
    // small frontiers go to the async mode; larger ones stay top-down
    const int64_t av = r.async_v, ae = r.async_e;
    auto small = [av, ae](int64_t qc, int64_t qe) { return qc <= av && qe <= ae; };

    for (int guard = 0; guard < (1 << 30); ++guard) {
        const int cur = level & 1;
        const int s_cur = level % 3, s_nx = (level + 1) % 3, s_free = (level + 2) % 3;
        unsigned long long pk = __ldcg(r.qpk + s_cur);
        int64_t qcount = (int64_t)(pk & kCountMask), qedges = (int64_t)(pk >> kCountBits);
        if (blockIdx.x == 0 && tid == 0) {  // free the slot read two levels ago
            r.qpk[s_free] = 0ull;
            slots[s_free] = LvlSlot{0, 0, 0, 0};
        }
        int64_t nvis = 0, mnext = 0, mother = 0;
        if (mode == M_TD) {
            int64_t nchunks = (qedges + kChunk - 1) / kChunk;
            for (int64_t c = blockIdx.x; c < nchunks; c += gridDim.x)
                td_chunk<OffT, DIR>(r, d, c, nchunks, qcount, qedges, cur, r.qpk + s_nx, nvis, mnext, mother,
                                    tid, tdsm);
        } else if (mode == M_BU) {
            // the slot read at this level's start is free until it is
            // recycled two levels on: its spare word counts the BU groups
            bu_words<OffT, DIR>(r, d, gwarp, nwarps, &slots[s_cur].spare, nvis, mnext, mother);
        } else {
            async_round<OffT, DIR>(r, d, cur, qcount, r.qpk + s_nx, nvis, mnext, mother, asm_);
        }
        // publish this level's totals (one atomic per CTA)
        {
            int64_t tv = block_sum64(nvis, sh);
            int64_t tn = block_sum64(mnext, sh);
            int64_t to = block_sum64(mother, sh);
            if (tid == 0 && (tv || tn || to)) {
                atomicAdd(&slots[s_nx].nvis, (unsigned long long)tv);
                atomicAdd(&slots[s_nx].m_next, (unsigned long long)tn);
                atomicAdd(&slots[s_nx].m_other, (unsigned long long)to);
            }
        }
        if (!grid_sync(r.gsync, r.err)) return;
        if (blockIdx.x == 0 && tid == 0 && level < kTraceLevels) {  // diagnostics: level, mode, time
            long long *t = r.trace + ((long long)DIR * kTraceLevels + level) * 4;
            t[0] = mode;
            t[1] = (long long)__ldcg(&slots[s_nx].nvis);
            t[2] = (long long)(__ldcg(r.qpk + s_nx) >> kCountBits);
            t[3] = (long long)globaltimer();
        }

        // ---- identical decision in every CTA ----
        LvlSlot s;
        s.nvis = __ldcg(&slots[s_nx].nvis);
        s.m_next = __ldcg(&slots[s_nx].m_next);
        s.m_other = __ldcg(&slots[s_nx].m_other);
        const int64_t nf = (int64_t)s.nvis;
        total_vis += nf;
        ++level;
        m_unexpl -= (int64_t)s.m_next;
        const unsigned long long pn = __ldcg(r.qpk + s_nx);
        const int64_t qcn = (int64_t)(pn & kCountMask), qen = (int64_t)(pn >> kCountBits);
        if (mode == M_BU) {
            if (nf == 0) { mode = M_DONE; break; }
            if (nf < n_total / max(r.beta, 1) || level > r.gamma) {
                // leave bottom-up for good: queue the vertices found this level
                left_bu = true;
                rebuild_queue<OffT, DIR>(r, d, level & 1, r.qpk + (level % 3), gwarp, nwarps);
                if (!grid_sync(r.gsync, r.err)) return;
                const unsigned long long pr = __ldcg(r.qpk + (level % 3));
                const int64_t qcr = (int64_t)(pr & kCountMask), qer = (int64_t)(pr >> kCountBits);
                if (qcr == 0) { mode = M_DONE; break; }
                mode = small(qcr, qer) ? M_ASYNC : M_TD;
            }
        } else {
            // top-down and async rounds hand over through the queue; what an
            // async round leaves there (hubs, overflow) is expanded top-down
            if (qcn == 0) { mode = M_DONE; break; }
            if (mode == M_ASYNC)
                mode = M_TD;
            else if (!left_bu && qen > m_unexpl / max(r.alpha, 1))
                mode = M_BU;
            else
                mode = small(qcn, qen) ? M_ASYNC : M_TD;
        }
        if (level > r.V + 2) {  // every level claims a vertex; more levels is a bug
            if (tid == 0) atomicCAS(r.err, 0, kErrOverflow);
            return;
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        r.counters[DIR == 0 ? C_FW_LEVELS : C_BW_LEVELS] = (unsigned long long)level;
        if (DIR == 0) atomicAdd(r.counters + C_FW_SIZE, (unsigned long long)total_vis);
    }
}

// Exact degree sums of the reached sets (statistics only, on request):
// sum of out-degrees over F and of in-degrees over B.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_reach_degrees(Run<OffT> r) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    const int lane = lane_id();
    const int64_t gw = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int64_t nw = (int64_t)gridDim.x * kWarps;
    int64_t fo = 0, bi = 0;
    for (int64_t wi = gw; wi < r.W; wi += nw) {
        uint32_t f = r.F[wi], b = r.B[wi];
        if (!(f | b)) continue;
        int64_t v = wi * 32 + lane;
        if ((f >> lane) & 1u) fo += ld_off(r.fw_beg, v + 1) - ld_off(r.fw_beg, v);
        if ((b >> lane) & 1u) bi += ld_off(r.bw_beg, v + 1) - ld_off(r.bw_beg, v);
    }
    int64_t a = block_sum64(fo, sh), c = block_sum64(bi, sh);
    if (threadIdx.x == 0) {
        if (a) atomicAdd(r.counters + C_FW_XDEG, (unsigned long long)a);
        if (c) atomicAdd(r.counters + C_BW_XDEG, (unsigned long long)c);
    }
}

// Size and out+in degree sum of a worklist (statistics only, on request):
// the algorithmic bytes of the trim stages that read it.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_list_degrees(Run<OffT> r, const int32_t *wl,
                                                         const unsigned long long *n_wl, int slot_n, int slot_deg) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    const int64_t n = (int64_t)*n_wl;
    int64_t d = 0;
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        const int64_t v = wl[i];
        d += ld_off(r.fw_beg, v + 1) - ld_off(r.fw_beg, v) + ld_off(r.bw_beg, v + 1) - ld_off(r.bw_beg, v);
    }
    const int64_t t = block_sum64(d, sh);
    if (threadIdx.x == 0) {
        if (t) atomicAdd(r.counters + slot_deg, (unsigned long long)t);
        if (slot_n >= 0 && blockIdx.x == 0) r.counters[slot_n] = (unsigned long long)n;
    }
}

}  // namespace ispan

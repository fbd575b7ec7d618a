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
//        spread over many CTAs, a run of low-degree vertices shares one chunk.
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
// DIR 1 (backward): visit map B, restricted to F, expands in-edges.
#pragma once
#include "common.cuh"

namespace ispan {

constexpr int kBuLane = 16;          // edges a lane scans alone in bottom-up
constexpr int64_t kTailV = 2048;     // frontier size that enters the CTA-0 tail
constexpr int64_t kTailE = 32768;    // ... and frontier edges
constexpr int kTailMaxLevels = 4096; // tail levels before re-joining the grid

enum BfsMode : int { M_TD = 0, M_BU = 1, M_TAIL = 2, M_DONE = 3 };

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
            R = r.F; Vm = r.B;
        }
    }
    __device__ __forceinline__ int64_t xdeg(int64_t v) const { return ld_off(xbeg, v + 1) - ld_off(xbeg, v); }
    __device__ __forceinline__ int64_t odeg(int64_t v) const { return ld_off(obeg, v + 1) - ld_off(obeg, v); }
};

// Expand one chunk of the current queue (top-down).  All threads of the CTA
// call it.  Newly visited vertices go to the next queue; per-thread sums
// accumulate into nvis / msum_next / msum_other.
template <typename OffT, int DIR>
__device__ __forceinline__ void td_chunk(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int64_t c,
                                         int64_t nchunks, int64_t qcount, int64_t qedges, int cur,
                                         unsigned long long *pk_next, int64_t &nvis, int64_t &msum_next,
                                         int64_t &msum_other, int tid) {
    const int32_t *qv = r.qv[cur];
    const int64_t *qe = r.qe[cur];
    const int32_t *qc = r.qchunk[cur];
    int nx = cur ^ 1;
    int64_t e0 = c * kChunk;
    int64_t e1 = min(e0 + (int64_t)kChunk, qedges);
    int64_t s_lo = __ldcg(qc + c);
    int64_t s_hi = (c + 1 < nchunks) ? (int64_t)__ldcg(qc + c + 1) : qcount - 1;
    if (!ICHK(s_lo >= 0 && s_lo <= s_hi && s_hi < qcount, 20, (s_lo << 32) | (s_hi & 0xffffffff))) return;
    // each thread owns a run of consecutive virtual edges, so one binary
    // search per thread finds its first slot and the walk follows the queue
    constexpr int kPer = kChunk / kBlock;
    int64_t my0 = e0 + (int64_t)tid * kPer;
    int64_t slot = s_lo;
    if (my0 < e1) {
        int64_t lo = s_lo, hi = s_hi;
        while (lo < hi) {  // last slot with qe[slot] <= my0
            int64_t mid = (lo + hi + 1) >> 1;
            if (__ldcg(qe + mid) <= my0) lo = mid; else hi = mid - 1;
        }
        slot = lo;
    }
    int64_t slot_e0 = (my0 < e1) ? __ldcg(qe + slot) : 0;
    int64_t slot_e1 = (my0 < e1) ? ((slot + 1 < qcount) ? __ldcg(qe + slot + 1) : qedges) : 0;
    int64_t base = (my0 < e1) ? ld_off(d.xbeg, __ldcg(qv + slot)) : 0;
#pragma unroll 1
    for (int k = 0; k < kPer; ++k) {
        int64_t e = my0 + k;
        bool live = e < e1;
        int32_t w = -1;
        if (live) {
            while (e >= slot_e1) {  // advance to the slot that owns e
                if (!ICHK(slot + 1 < qcount, 21, slot)) break;
                ++slot;
                slot_e0 = slot_e1;
                slot_e1 = (slot + 1 < qcount) ? __ldcg(qe + slot + 1) : qedges;
                base = ld_off(d.xbeg, __ldcg(qv + slot));
            }
            w = ld_adj(d.xadj, base + (e - slot_e0));
        }
        bool nw = false;
        if (live && bit(d.R, w) && !bitv(d.Vm, w)) nw = set_bit(d.Vm, w);
        int64_t dg = nw ? d.xdeg(w) : 0;
        if (nw) {
            nvis += 1;
            msum_next += dg;
            msum_other += d.odeg(w);
        }
        q_append(nw, w, dg, r.qv[nx], r.qe[nx], r.qchunk[nx], pk_next, r.V);
    }
}

// Bottom-up over bitmap words [w_lo, w_hi) with warp stride.
template <typename OffT, int DIR>
__device__ __forceinline__ void bu_words(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int64_t w_begin,
                                         int64_t w_stride, int64_t &nvis, int64_t &msum_next,
                                         int64_t &msum_other) {
    const int lane = lane_id();
    for (int64_t wi = w_begin; wi < r.W; wi += w_stride) {
        uint32_t vis = *((volatile uint32_t *)(d.Vm + wi));
        uint32_t cand = __ldg(d.R + wi) & ~vis;
        if (lane == 0) r.P[wi] = vis;  // snapshot for a later switch to top-down
        if (!cand) continue;
        int64_t v = wi * 32 + lane;
        bool mine = (cand >> lane) & 1u;
        bool found = false, rem = false;
        int64_t e = 0, end = 0;
        if (mine) {
            e = ld_off(d.pbeg, v);
            end = ld_off(d.pbeg, v + 1);
            int64_t cap = min(end, e + (int64_t)kBuLane);
            for (; e < cap; ++e)
                if (bitv(d.Vm, ld_adj(d.padj, e))) { found = true; break; }
            rem = !found && e < end;
        }
        unsigned rm = __ballot_sync(kFull, rem);
        while (rm) {  // the warp finishes long scans one lane at a time
            int l = __ffs(rm) - 1;
            rm &= rm - 1;
            int64_t le = __shfl_sync(kFull, e, l), lend = __shfl_sync(kFull, end, l);
            bool hit = false;
            for (int64_t b = le; b < lend; b += 32) {
                int64_t i = b + lane;
                bool h = i < lend && bitv(d.Vm, ld_adj(d.padj, i));
                if (__any_sync(kFull, h)) { hit = true; break; }
            }
            if (lane == l) found = hit;
        }
        unsigned fm = __ballot_sync(kFull, found);
        if (fm && lane == 0) atomicOr(d.Vm + wi, fm);
        if (found) {
            nvis += 1;
            msum_next += d.xdeg(v);
            msum_other += d.odeg(v);
        }
    }
}

// Rebuild the top-down queue from the vertices visited during the last
// bottom-up level (visit map minus its snapshot).
template <typename OffT, int DIR>
__device__ __forceinline__ void rebuild_queue(const Run<OffT> &r, const BfsDir<OffT, DIR> &d, int nx,
                                              unsigned long long *pk, int64_t w_begin, int64_t w_stride) {
    const int lane = lane_id();
    for (int64_t wi = w_begin; wi < r.W; wi += w_stride) {
        uint32_t nw = __ldcg(d.Vm + wi) & ~__ldcg(r.P + wi);
        bool me = (nw >> lane) & 1u;
        int64_t v = wi * 32 + lane;
        int64_t dg = me ? d.xdeg(v) : 0;
        q_append(me, (int32_t)v, dg, r.qv[nx], r.qe[nx], r.qchunk[nx], pk, r.V);
    }
}

template <typename OffT, int DIR>
__global__ void __launch_bounds__(kBlock) k_bfs(Run<OffT> r, BfsCtl *ctl) {
    __shared__ int64_t sh[kWarps];
    const BfsDir<OffT, DIR> d(r);
    const int tid = threadIdx.x;
    const int64_t gwarp = ((int64_t)blockIdx.x * kBlock + tid) >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * kWarps;
    LvlSlot *slots = reinterpret_cast<LvlSlot *>(r.lvl);

    // budget for the alpha rule: unexplored expansion-side edges
    int64_t m_unexpl = (int64_t)(DIR == 0 ? r.counters[C_MU0] : r.counters[C_FW_MU]);
    const int64_t n_total = (int64_t)(DIR == 0 ? r.counters[C_ACTIVE0] : r.counters[C_FW_SIZE]);
    int level = 0, mode = M_TD;
    int64_t total_vis = 0;

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
                                    tid);
        } else if (mode == M_BU) {
            bu_words<OffT, DIR>(r, d, gwarp, nwarps, nvis, mnext, mother);
        } else if (mode == M_TAIL) {
            if (blockIdx.x == 0) {
                // CTA 0 alone: levels separated by __syncthreads only
                int lv = level, exit_mode = M_DONE;
                int64_t tv_all = 0, tm_all = 0, tx_all = 0;
                for (int it = 0; it < kTailMaxLevels; ++it) {
                    const int c2 = lv & 1;
                    const int sc = lv % 3, sn = (lv + 1) % 3, sf = (lv + 2) % 3;
                    unsigned long long p2 = __ldcg(r.qpk + sc);
                    int64_t qc2 = (int64_t)(p2 & kCountMask), qe2 = (int64_t)(p2 >> kCountBits);
                    if (tid == 0) r.qpk[sf] = 0ull;
                    __syncthreads();
                    int64_t nv = 0, m1 = 0, m2 = 0;
                    int64_t nch = (qe2 + kChunk - 1) / kChunk;
                    for (int64_t c = 0; c < nch; ++c)
                        td_chunk<OffT, DIR>(r, d, c, nch, qc2, qe2, c2, r.qpk + sn, nv, m1, m2, tid);
                        tv_all += block_sum64(nv, sh);
                    tm_all += block_sum64(m2, sh);
                    tx_all += block_sum64(m1, sh);
                    ++lv;
                    unsigned long long pn = __ldcg(r.qpk + sn);
                    int64_t qcn = (int64_t)(pn & kCountMask), qen = (int64_t)(pn >> kCountBits);
                    if (qcn == 0) { exit_mode = M_DONE; break; }
                    if (qcn > 4 * kTailV || qen > 4 * kTailE) { exit_mode = M_TD; break; }
                    exit_mode = M_TAIL;  // still small after kTailMaxLevels: re-join, then resume
                }
                if (tid == 0) {
                    total_vis += tv_all;
                    if (DIR == 0 && tm_all) atomicAdd(r.counters + C_FW_MU, (unsigned long long)tm_all);
                    if (tx_all) atomicAdd(r.counters + (DIR == 0 ? C_FW_XDEG : C_BW_XDEG), (unsigned long long)tx_all);
                    for (int i = 0; i < 3; ++i) slots[i] = LvlSlot{0, 0, 0, 0};
                    ctl->level = lv;
                    ctl->mode = exit_mode;
                }
            }
        }
        // publish this level's totals (one atomic per CTA)
        if (mode != M_TAIL) {
            int64_t tv = block_sum64(nvis, sh);
            int64_t tn = block_sum64(mnext, sh);
            int64_t to = block_sum64(mother, sh);
            if (tid == 0 && tv) {
                atomicAdd(&slots[s_nx].nvis, (unsigned long long)tv);
                atomicAdd(&slots[s_nx].m_next, (unsigned long long)tn);
                atomicAdd(&slots[s_nx].m_other, (unsigned long long)to);
            }
        }
        if (!grid_sync(r.gsync, r.err)) return;

        // ---- identical decision in every CTA ----
        if (mode == M_TAIL) {
            level = __ldcg(&ctl->level);
            mode = __ldcg(&ctl->mode);
            if (mode == M_DONE) break;
            continue;  // M_TD: the tail's last queue is the current level's; M_TAIL: resume
        }
        LvlSlot s;
        s.nvis = __ldcg(&slots[s_nx].nvis);
        s.m_next = __ldcg(&slots[s_nx].m_next);
        s.m_other = __ldcg(&slots[s_nx].m_other);
        int64_t nf = (int64_t)s.nvis;
        total_vis += nf;
        if (DIR == 0 && blockIdx.x == 0 && tid == 0 && s.m_other)
            atomicAdd(r.counters + C_FW_MU, s.m_other);
        if (blockIdx.x == 0 && tid == 0 && s.m_next)
            atomicAdd(r.counters + (DIR == 0 ? C_FW_XDEG : C_BW_XDEG), s.m_next);
        ++level;
        if (nf == 0) { mode = M_DONE; break; }
        m_unexpl -= (int64_t)s.m_next;
        if (mode == M_TD) {
            unsigned long long pn = __ldcg(r.qpk + s_nx);
            int64_t qcn = (int64_t)(pn & kCountMask), qen = (int64_t)(pn >> kCountBits);
            if (qen > m_unexpl / max(r.alpha, 1)) {
                mode = M_BU;
            } else if (qcn <= kTailV && qen <= kTailE) {
                mode = M_TAIL;
                if (blockIdx.x == 0 && tid == 0) { ctl->level = level; ctl->mode = M_TAIL; }
            }
        } else {  // bottom-up
            if (nf < n_total / max(r.beta, 1) || level > r.gamma) {
                // leave bottom-up for good: queue the vertices found this level
                rebuild_queue<OffT, DIR>(r, d, level & 1, r.qpk + (level % 3), gwarp, nwarps);
                if (!grid_sync(r.gsync, r.err)) return;
                mode = M_TD;
                unsigned long long pn = __ldcg(r.qpk + (level % 3));
                int64_t qcn = (int64_t)(pn & kCountMask), qen = (int64_t)(pn >> kCountBits);
                if (qcn <= kTailV && qen <= kTailE) {
                    mode = M_TAIL;
                    if (blockIdx.x == 0 && tid == 0) { ctl->level = level; ctl->mode = M_TAIL; }
                }
            }
        }
    }
    if (blockIdx.x == 0 && tid == 0) {
        r.counters[DIR == 0 ? C_FW_LEVELS : C_BW_LEVELS] = (unsigned long long)level;
        if (DIR == 0) atomicAdd(r.counters + C_FW_SIZE, (unsigned long long)total_vis);
    }
}

}  // namespace ispan

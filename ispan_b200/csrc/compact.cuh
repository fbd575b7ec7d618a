// compact.cuh -- the compact graph the colouring of large WCCs runs on.
//
// The colouring rounds (k_color, stages.cuh) work on the vertices of the
// large WCCs only: on web-shaped graphs ~15 % of the vertices, with a quarter
// of their edges leading outside them (to the giant SCC, the trimmed
// sources and sinks).  On the input graph every edge check reads a colour
// word indexed over the whole vertex range and rejects the outside
// neighbours by their class; the offsets and adjacency are read over the
// whole CSR.  Here, before the rounds start, those vertices get dense ids
// 0..n-1 (their order in the large-WCC list, i.e. about the input order) and
// their edges among themselves are copied into a CSR of those ids, in the
// context's scratch that is free at this point:
//   compact id -> original id   x.small      (int32, n)
//   original id -> compact id   r.cnt_out    (int32, valid where A is set)
//   out/in degrees              r.members, x.roots
//   offsets (int32)             r.qe[1] viewed as int32: out at [0, n], in at [V+1, V+1+n]
//   adjacency (int32)           r.wl[0..1] (out), r.members..x.roots (in, written once the
//                               degrees there are scanned); each pair is one block of 2 V
// so the random accesses of the rounds fall on n colour words instead of V,
// and no edge check lands on a vertex outside.  The graph is built only when
// each direction's edges fit the adjacency arrays (at most V entries, int32
// offsets); otherwise K_CMP_OK stays 0 and the colouring runs on the input
// graph.  Membership is the active map A: at this point exactly the vertices
// of the large WCCs are active.  The fill kernel reads only the offsets, so
// the in-adjacency may overwrite the degree arrays.
#pragma once
#include "stages.cuh"

namespace ispan {

constexpr int kScanBlocks = 1024;  // blocks of the offset scans (at most; one CTA scans their sums)
constexpr int64_t kCmpMin = 1 << 16;  // fewer colouring vertices than this: no compact graph (the
                                      // input graph's colour words of so few vertices stay in L2)

// Whether the compact graph is worth building: enough colouring vertices,
// and spread thinly over the id range (at most a quarter of it).  Where they
// are dense -- a batch, whose graphs are contiguous id ranges -- the input
// graph's words and lists are already local, and measured on the batched
// workload the build cost more than the rounds gained.
__device__ __forceinline__ bool cmp_wanted(int64_t n, int64_t V) { return n >= kCmpMin && 4 * n <= V; }

struct CmpBufs {
    int32_t *newid;   // [V]
    int32_t *old;     // [n]
    int32_t *dout, *din;
    int32_t *fbeg, *bbeg;  // [n + 1] each
    int32_t *fadj, *badj;  // [cap_e] each
    long long *bsum;       // [2 * kScanBlocks]
    int64_t cap_e;         // adjacency capacity per direction
    int64_t V;             // vertices of the input graph
};

// ids (compact id i <-> original id L[i]), active out- and in-degrees
// (self-loops dropped), and the per scan block sums of the degrees
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cmp_count(Run<OffT> r, Ext<OffT> x, CmpBufs b) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t sh[kWarps];
    const int64_t n = (int64_t)__ldcg(x.ctl + K_LARGE);
    if (!cmp_wanted(n, b.V)) return;
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = min(n, (int64_t)blockIdx.x * per), i1 = min(n, i0 + per);
    int64_t so = 0, si = 0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += kBlock) {
        const int32_t v = x.large[0][i];
        b.newid[v] = (int32_t)i;
        b.old[i] = v;
        int32_t co = 0, ci = 0;
        for (int64_t e = ld_off(r.fw_beg, v), e1 = ld_off(r.fw_beg, v + 1); e < e1; ++e) {
            const int32_t w = ld_adj(r.fw_adj, e);
            co += (w != v) && bitc(r.A, w);
        }
        for (int64_t e = ld_off(r.bw_beg, v), e1 = ld_off(r.bw_beg, v + 1); e < e1; ++e) {
            const int32_t w = ld_adj(r.bw_adj, e);
            ci += (w != v) && bitc(r.A, w);
        }
        b.dout[i] = co;
        b.din[i] = ci;
        so += co;
        si += ci;
    }
    const int64_t to = block_sum64(so, sh), ti = block_sum64(si, sh);
    if (threadIdx.x == 0) {
        b.bsum[blockIdx.x] = to;
        b.bsum[kScanBlocks + blockIdx.x] = ti;
    }
}

// one CTA of kScanBlocks threads: exclusive scan of the block sums (a
// thread per block sum, warp scans, then the warp totals); the graph is
// built only if both directions fit
__global__ void __launch_bounds__(kScanBlocks) k_cmp_tops(unsigned long long *ctl, CmpBufs b, int nblk) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ long long wt[2][kScanBlocks / 32];
    const int64_t n = (int64_t)__ldcg(ctl + K_LARGE);
    if (!cmp_wanted(n, b.V)) {
        if (threadIdx.x == 0) ctl[K_CMP_OK] = 0ull;
        return;
    }
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    long long v[2], incl[2];
    for (int d = 0; d < 2; ++d) {
        v[d] = t < nblk ? b.bsum[d * kScanBlocks + t] : 0;
        incl[d] = v[d];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(kFull, incl[d], o);
            if (lane >= o) incl[d] += y;
        }
        if (lane == 31) wt[d][warp] = incl[d];
    }
    __syncthreads();
    if (warp == 0) {
        for (int d = 0; d < 2; ++d) {
            long long x = wt[d][lane], xi = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(kFull, xi, o);
                if (lane >= o) xi += y;
            }
            wt[d][lane] = xi - x;  // exclusive base of each warp
            if (lane == 31) {
                if (d == 0) ctl[K_CMP_EF] = (unsigned long long)xi;
                else ctl[K_CMP_EB] = (unsigned long long)xi;
            }
        }
    }
    __syncthreads();
    for (int d = 0; d < 2; ++d)
        if (t < nblk) b.bsum[d * kScanBlocks + t] = wt[d][warp] + incl[d] - v[d];
    if (t == 0) {
        const long long o = (long long)ctl[K_CMP_EF], in = (long long)ctl[K_CMP_EB];
        const bool fits = o <= b.cap_e && in <= b.cap_e && o < INT32_MAX && in < INT32_MAX;
        ctl[K_CMP_OK] = fits ? 1ull : 0ull;
    }
}

// offsets: each block rescans its range from its base (serial per thread
// over a contiguous sub-range, then a block scan of the thread totals)
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cmp_offsets(Run<OffT> r, Ext<OffT> x, CmpBufs b) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ int64_t st[kBlock];
    if (!__ldcg(x.ctl + K_CMP_OK)) return;
    const int64_t n = (int64_t)__ldcg(x.ctl + K_LARGE);
    const int64_t per = (n + gridDim.x - 1) / gridDim.x;
    const int64_t i0 = min(n, (int64_t)blockIdx.x * per), i1 = min(n, i0 + per);
    const int64_t sub = (i1 - i0 + kBlock - 1) / kBlock;
    const int64_t j0 = min(i1, i0 + threadIdx.x * sub), j1 = min(i1, j0 + sub);
    for (int dir = 0; dir < 2; ++dir) {
        const int32_t *deg = dir ? b.din : b.dout;
        int32_t *beg = dir ? b.bbeg : b.fbeg;
        int64_t t = 0;
        for (int64_t j = j0; j < j1; ++j) t += deg[j];
        st[threadIdx.x] = t;
        __syncthreads();
        if (threadIdx.x == 0) {  // 512 entries, once per block and direction
            int64_t run = b.bsum[dir * kScanBlocks + blockIdx.x];
            for (int k = 0; k < kBlock; ++k) {
                const int64_t y = st[k];
                st[k] = run;
                run += y;
            }
        }
        __syncthreads();
        int64_t run = st[threadIdx.x];
        for (int64_t j = j0; j < j1; ++j) {
            beg[j] = (int32_t)run;
            run += deg[j];
        }
        if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
            beg[n] = (int32_t)__ldcg(x.ctl + (dir ? K_CMP_EB : K_CMP_EF));
        __syncthreads();
    }
}

// adjacency in compact ids (input order kept), and the large-WCC list in
// compact ids
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cmp_fill(Run<OffT> r, Ext<OffT> x, CmpBufs b) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    if (!__ldcg(x.ctl + K_CMP_OK)) return;
    const int64_t n = (int64_t)__ldcg(x.ctl + K_LARGE);
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        const int32_t v = b.old[i];
        int64_t p = b.fbeg[i];
        for (int64_t e = ld_off(r.fw_beg, v), e1 = ld_off(r.fw_beg, v + 1); e < e1; ++e) {
            const int32_t w = ld_adj(r.fw_adj, e);
            if (w != v && bitc(r.A, w)) b.fadj[p++] = __ldcg(b.newid + w);
        }
        p = b.bbeg[i];
        for (int64_t e = ld_off(r.bw_beg, v), e1 = ld_off(r.bw_beg, v + 1); e < e1; ++e) {
            const int32_t w = ld_adj(r.bw_adj, e);
            if (w != v && bitc(r.A, w)) b.badj[p++] = __ldcg(b.newid + w);
        }
        x.large[0][i] = (int32_t)i;
    }
}

}  // namespace ispan

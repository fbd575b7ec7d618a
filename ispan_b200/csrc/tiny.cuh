// tiny.cuh -- every stage after the giant SCC for a small residual, in one CTA.
//
// On small graphs (R-MAT scale 16: 65,536 vertices, ~1 M edges) the pivot
// SCC and the first trim leave a residual of tens of vertices, and each of
// the dozen stage kernels that follow (two peels, trim-2, trim-3, the eight
// WCC launches, the small-WCC kernel, the colouring) costs its launch and,
// for the persistent ones, grid barriers -- about 100 us for no work.  When
// at most kTinyV vertices remain, with at most kTinyE edges among them in
// each direction, k_tiny_residual copies their induced subgraph into shared
// memory (local ids through the aux2 scratch array, free until the WCC
// stage) and runs the same sequence there:
//   1. trim-1 to a fixpoint (the peel of src/trim_1_gfq.h:365-458): a vertex
//      with no live in- or out-edge is its own SCC; counters drop as
//      neighbours go, by edge (duplicates count, as in k_trim1);
//   2. trim-2 (src/trim_2_3.h:146-283) and 3. trim-3 (:482-1080) with the
//      patterns of k_trim2 / k_trim3 over distinct live neighbours, one
//      thread per vertex, claims by an atomic on a shared bitmap;
//   4. trim-1 again;
//   5. the rest: weakly connected components (statistics, as the WCC
//      stage counts them) and an iterative Tarjan, as k_local_scc does for
//      a small WCC.
// Labels are the minimum member id, classes as the stage kernels set them,
// counters and histogram entries as they record them, and every vertex
// leaves the active map.  It then sets K_TINY, and the later stage kernels
// return at once.  If the residual is larger, it returns without a trace
// (aux2 entries it wrote are rewritten before the WCC stage reads them).
#pragma once
#include "stages.cuh"

namespace ispan {

constexpr int kTinyV = 1024;  // residual vertices handled in shared memory ...
constexpr int kTinyE = 4096;  // ... and edges among them, per direction

struct TinySmem {
    int32_t gid[kTinyV];                 // local id -> vertex id
    int32_t ooff[kTinyV + 1], ioff[kTinyV + 1];
    uint16_t oadj[kTinyE], iadj[kTinyE];  // local ids
    int32_t co[kTinyV], ci[kTinyV];      // peel counters; then WCC labels (co) and Tarjan edge cursors (ci)
    uint32_t dead[kTinyV / 32];          // assigned to an SCC
    uint32_t fresh[kTinyV / 32];         // peeled in the current round
    int16_t idx[kTinyV], low[kTinyV], stk[kTinyV], csv[kTinyV];
    uint8_t onst[kTinyV];
    int32_t wsum[kBlock / 32];
    int flag, n_peel, n_t2, n_t3, rounds;
};

__device__ __forceinline__ bool tiny_dead(const TinySmem &s, int i) { return (s.dead[i >> 5] >> (i & 31)) & 1u; }
__device__ __forceinline__ bool tiny_claim(TinySmem &s, int i) {
    const uint32_t b = 1u << (i & 31);
    return !(atomicOr(&s.dead[i >> 5], b) & b);
}

// exclusive prefix of a[0..n) in place, total in a[n]; all threads call it
__device__ __forceinline__ void tiny_scan(int32_t *a, int n, TinySmem &s) {
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (n + kBlock - 1) / kBlock;  // consecutive entries per thread (2 for n = 1024)
    const int j0 = min(n, t * per), j1 = min(n, j0 + per);
    int sum = 0;
    for (int j = j0; j < j1; ++j) sum += a[j];
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s.wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int w = lane < kBlock / 32 ? s.wsum[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kBlock / 32) s.wsum[lane] = wi - w;
        if (lane == 31) a[n] = wi;  // (kBlock / 32 <= 32 warps: lane 31 holds the total)
    }
    __syncthreads();
    int run = s.wsum[warp] + incl - sum;
    for (int j = j0; j < j1; ++j) {
        const int y = a[j];
        a[j] = run;
        run += y;
    }
    __syncthreads();
}

// trim-1 to a fixpoint over the live vertices; returns the rounds taken
template <typename OffT>
__device__ int tiny_peel(const Run<OffT> &r, TinySmem &s, int n) {
    const int t = threadIdx.x;
    for (int i = t; i < n; i += kBlock) {  // live edge counts (duplicates count, self-loops do not exist here)
        if (tiny_dead(s, i)) continue;
        int o = 0, c = 0;
        for (int e = s.ooff[i]; e < s.ooff[i + 1]; ++e) o += !tiny_dead(s, s.oadj[e]);
        for (int e = s.ioff[i]; e < s.ioff[i + 1]; ++e) c += !tiny_dead(s, s.iadj[e]);
        s.co[i] = o;
        s.ci[i] = c;
    }
    __syncthreads();
    int rounds = 0;
    for (int guard = 0; guard <= kTinyV + 1; ++guard) {
        if (t == 0) s.flag = 0;
        for (int i = t; i < kTinyV / 32; i += kBlock) s.fresh[i] = 0u;
        __syncthreads();
        for (int i = t; i < n; i += kBlock) {
            if (tiny_dead(s, i) || (s.co[i] > 0 && s.ci[i] > 0)) continue;
            atomicOr(&s.fresh[i >> 5], 1u << (i & 31));
            s.flag = 1;
        }
        __syncthreads();
        const int any = s.flag;
        if (!any) break;
        ++rounds;
        for (int i = t; i < n; i += kBlock)  // this round's vertices leave, each its own SCC
            if ((s.fresh[i >> 5] >> (i & 31)) & 1u) {
                atomicOr(&s.dead[i >> 5], 1u << (i & 31));
                const int32_t v = s.gid[i];
                r.label[v] = v;
                r.cls[v] = CLS_TRIM1;
                atomicAdd(&s.n_peel, 1);
            }
        __syncthreads();
        for (int i = t; i < n; i += kBlock) {  // their live neighbours lose an edge each
            if (!((s.fresh[i >> 5] >> (i & 31)) & 1u)) continue;
            for (int e = s.ooff[i]; e < s.ooff[i + 1]; ++e)
                if (!tiny_dead(s, s.oadj[e])) atomicSub(&s.ci[s.oadj[e]], 1);
            for (int e = s.ioff[i]; e < s.ioff[i + 1]; ++e)
                if (!tiny_dead(s, s.iadj[e])) atomicSub(&s.co[s.iadj[e]], 1);
        }
        __syncthreads();
    }
    return rounds + 1;  // the last, empty round counts as in k_trim1
}

// up to `cap` distinct live neighbours of i in one direction, skipping x1, x2
__device__ __forceinline__ int tiny_distinct(const TinySmem &s, const int32_t *off, const uint16_t *adj, int i,
                                             int x1, int x2, int cap, int &n1, int &n2) {
    int d = 0;
    for (int e = off[i]; e < off[i + 1] && d < cap; ++e) {
        const int w = adj[e];
        if (w == x1 || w == x2 || tiny_dead(s, w)) continue;
        if (d == 0) { n1 = w; d = 1; }
        else if (d == 1 && w != n1) { n2 = w; d = 2; }
        else if (d == 2 && w != n1 && w != n2) { d = 3; }
    }
    return d;
}

// claim a 2- or 3-vertex pattern: the first claim decides (another thread
// that found the same set claims nothing more); label = min member id
template <typename OffT>
__device__ __forceinline__ int tiny_take(const Run<OffT> &r, TinySmem &s, const int *m, int k, uint8_t cls) {
    int32_t lab = INT32_MAX;
    for (int q = 0; q < k; ++q) lab = min(lab, s.gid[m[q]]);
    int got = 0;
    for (int q = 0; q < k; ++q)
        if (tiny_claim(s, m[q])) {
            r.label[s.gid[m[q]]] = lab;
            r.cls[s.gid[m[q]]] = cls;
            ++got;
        }
    return got;
}

template <typename OffT>
__device__ void tiny_trim23(const Run<OffT> &r, TinySmem &s, int n, int size) {
    for (int i = threadIdx.x; i < n; i += kBlock) {
        if (tiny_dead(s, i)) continue;
        for (int dir = 0; dir < 2; ++dir) {
            const int32_t *off = dir == 0 ? s.ooff : s.ioff;
            const uint16_t *adj = dir == 0 ? s.oadj : s.iadj;
            int a = -1, b = -1, y = -1, z = -1;
            if (size == 2) {  // i's only live neighbour a has i as its only live neighbour
                if (tiny_distinct(s, off, adj, i, i, i, 2, a, b) != 1) continue;
                if (tiny_distinct(s, off, adj, a, a, a, 2, y, z) != 1 || y != i) continue;
                const int m[2] = {i, a};
                atomicAdd(&s.n_t2, tiny_take(r, s, m, 2, CLS_TRIM2));
                break;
            }
            const int nv = tiny_distinct(s, off, adj, i, i, i, 3, a, b);
            int m[3];
            if (nv == 1) {  // cycle: i -> a -> c -> i
                if (tiny_distinct(s, off, adj, a, a, i, 2, y, z) != 1) continue;
                const int c = y;
                if (tiny_distinct(s, off, adj, c, c, a, 2, y, z) != 1 || y != i) continue;
                m[0] = i; m[1] = a; m[2] = c;
            } else if (nv == 2) {  // hub: i <-> a, i <-> b
                if (tiny_distinct(s, off, adj, a, a, b, 2, y, z) != 1 || y != i) continue;
                if (tiny_distinct(s, off, adj, b, b, a, 2, y, z) != 1 || y != i) continue;
                m[0] = i; m[1] = a; m[2] = b;
            } else {
                continue;
            }
            atomicAdd(&s.n_t3, tiny_take(r, s, m, 3, CLS_TRIM3));
            break;
        }
    }
    __syncthreads();
}

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_tiny_residual(Run<OffT> r, Ext<OffT> x) {
    pdl_wait();  // predecessor done, its writes visible
    pdl_trigger();
    __shared__ TinySmem s;
    const int t = threadIdx.x;
    const int64_t n64 = (int64_t)__ldcg(x.ctl + K_WL0);
    if (n64 > kTinyV) return;  // the stage kernels take it
    const int n = (int)n64;
    const int32_t *wl = r.wl[0];
    int32_t *lid = r.aux2;  // vertex id -> local id (the residual's vertices only)
    for (int i = t; i < n; i += kBlock) {
        const int32_t v = wl[i];
        s.gid[i] = v;
        lid[v] = i;
    }
    for (int i = t; i < kTinyV / 32; i += kBlock) s.dead[i] = 0u;
    if (t == 0) { s.n_peel = 0; s.n_t2 = 0; s.n_t3 = 0; }
    __syncthreads();
    // edges among the residual's vertices (the active map is exactly the
    // residual now), counted, then scanned, then copied in local ids: a warp
    // per vertex, its lanes striding the list (residual vertices can be hubs
    // whose lists run to thousands of edges, mostly into the removed giant)
    const int lane = t & 31, warp = t >> 5;
    for (int i = warp; i < n; i += kWarps) {
        const int32_t v = s.gid[i];
        int cnt[2];
        for (int dir = 0; dir < 2; ++dir) {
            const OffT *beg = dir == 0 ? r.fw_beg : r.bw_beg;
            const int32_t *adj = dir == 0 ? r.fw_adj : r.bw_adj;
            int c = 0;
            for (int64_t e = ld_off(beg, v) + lane, e1 = ld_off(beg, v + 1); e < e1; e += 32) {
                const int32_t w = ld_adj(adj, e);
                c += w != v && bitc(r.A, w);
            }
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
            cnt[dir] = c;
        }
        if (lane == 0) {
            s.ooff[i] = cnt[0];
            s.ioff[i] = cnt[1];
        }
    }
    __syncthreads();
    tiny_scan(s.ooff, n, s);
    tiny_scan(s.ioff, n, s);
    if (s.ooff[n] > kTinyE || s.ioff[n] > kTinyE) return;  // uniform: every thread reads the same totals
    for (int i = warp; i < n; i += kWarps) {
        const int32_t v = s.gid[i];
        for (int dir = 0; dir < 2; ++dir) {
            const OffT *beg = dir == 0 ? r.fw_beg : r.bw_beg;
            const int32_t *adj = dir == 0 ? r.fw_adj : r.bw_adj;
            uint16_t *ladj = dir == 0 ? s.oadj : s.iadj;
            int p = dir == 0 ? s.ooff[i] : s.ioff[i];
            const int64_t e0 = ld_off(beg, v), e1 = ld_off(beg, v + 1);
            for (int64_t b = e0; b < e1; b += 32) {  // warp-uniform steps; kept edges in list order
                const int64_t e = b + lane;
                const int32_t w = e < e1 ? ld_adj(adj, e) : v;
                const bool keep = w != v && bitc(r.A, w);
                const unsigned m = __ballot_sync(kFull, keep);
                const int at = p + __popc(m & lanemask_lt());
                if (keep && ICHK(at < kTinyE, 19, at)) ladj[at] = (uint16_t)__ldcg(lid + w);
                p += __popc(m);
            }
        }
    }
    __syncthreads();
    // the stage sequence of the pipeline, in shared memory
    int rounds = tiny_peel(r, s, n);
    tiny_trim23(r, s, n, 2);
    tiny_trim23(r, s, n, 3);
    rounds += tiny_peel(r, s, n);
    // what is left: weakly connected components (counted as the WCC stage
    // counts them), by min-label propagation over the live edges
    int32_t *wcc = s.co;
    for (int i = t; i < n; i += kBlock) wcc[i] = i;
    __syncthreads();
    for (int guard = 0; guard <= kTinyV; ++guard) {
        __syncthreads();  // every thread has read the last round's flag
        if (t == 0) s.flag = 0;
        __syncthreads();
        for (int i = t; i < n; i += kBlock) {
            if (tiny_dead(s, i)) continue;
            int m = wcc[i];
            for (int e = s.ooff[i]; e < s.ooff[i + 1]; ++e)
                if (!tiny_dead(s, s.oadj[e])) m = min(m, wcc[s.oadj[e]]);
            for (int e = s.ioff[i]; e < s.ioff[i + 1]; ++e)
                if (!tiny_dead(s, s.iadj[e])) m = min(m, wcc[s.iadj[e]]);
            if (m < wcc[i]) {
                atomicMin(&wcc[i], m);
                s.flag = 1;
            }
        }
        __syncthreads();
        if (!s.flag) break;
    }
    // Tarjan (one thread, as k_local_scc) over the live vertices
    if (t == 0) {
        int nwcc = 0, nmice = 0, nscc = 0;
        for (int i = 0; i < n; ++i) {
            s.idx[i] = -1;
            s.onst[i] = 0;
            if (!tiny_dead(s, i)) {
                nwcc += wcc[i] == i;
                ++nmice;
            }
        }
        int counter = 0, sp = 0;
        int32_t *cse = s.ci;
        for (int s0 = 0; s0 < n; ++s0) {
            if (s.idx[s0] != -1 || tiny_dead(s, s0)) continue;
            int cp = 1;
            s.csv[0] = (int16_t)s0;
            cse[0] = s.ooff[s0];
            s.idx[s0] = s.low[s0] = (int16_t)counter++;
            s.stk[sp++] = (int16_t)s0;
            s.onst[s0] = 1;
            while (cp > 0) {
                const int vv = s.csv[cp - 1];
                int e = cse[cp - 1];
                bool down = false;
                for (; e < s.ooff[vv + 1]; ++e) {
                    const int w = s.oadj[e];
                    if (tiny_dead(s, w)) continue;
                    if (s.idx[w] == -1) {
                        cse[cp - 1] = e + 1;
                        s.idx[w] = s.low[w] = (int16_t)counter++;
                        s.stk[sp++] = (int16_t)w;
                        s.onst[w] = 1;
                        s.csv[cp] = (int16_t)w;
                        cse[cp] = s.ooff[w];
                        ++cp;
                        down = true;
                        break;
                    } else if (s.onst[w] && s.idx[w] < s.low[vv]) {
                        s.low[vv] = s.idx[w];
                    }
                }
                if (down) continue;
                if (s.low[vv] == s.idx[vv]) {
                    int32_t mn = INT32_MAX;
                    int k = sp, sz = 0;
                    do {
                        --k;
                        mn = min(mn, s.gid[s.stk[k]]);
                        ++sz;
                    } while (s.stk[k] != vv);
                    while (sp > k) {
                        const int w = s.stk[--sp];
                        s.onst[w] = 0;
                        r.label[s.gid[w]] = mn;
                        r.cls[s.gid[w]] = CLS_MICE;
                    }
                    atomicAdd((unsigned long long *)(r.hist + sz), 1ull);  // sz <= kTinyV < kHistCap
                    ++nscc;
                }
                --cp;
                if (cp > 0) {
                    const int p = s.csv[cp - 1];
                    if (s.low[vv] < s.low[p]) s.low[p] = s.low[vv];
                }
            }
        }
        if (s.n_peel) atomicAdd(r.counters + C_TRIM1, (unsigned long long)s.n_peel);
        if (s.n_t2) atomicAdd(r.counters + C_TRIM2, (unsigned long long)s.n_t2);
        if (s.n_t3) atomicAdd(r.counters + C_TRIM3, (unsigned long long)s.n_t3);
        if (nmice) {
            atomicAdd(r.counters + C_MICE_V, (unsigned long long)nmice);
            atomicAdd(r.counters + C_MICE_SCC, (unsigned long long)nscc);
        }
        if (nwcc) {
            atomicAdd(r.counters + C_WCC, (unsigned long long)nwcc);
            atomicAdd(r.counters + C_LOCAL_WCC, (unsigned long long)nwcc);
        }
        atomicAdd(r.counters + C_TRIM_ROUNDS, (unsigned long long)rounds);
    }
    __syncthreads();
    // every residual vertex has its SCC: all leave the active map
    for (int i = t; i < n; i += kBlock) clear_bit(r.A, s.gid[i]);
    __syncthreads();
    if (t == 0) {
        __threadfence();
        x.ctl[K_TINY] = 1ull;  // the later stage kernels return at once
    }
}

}  // namespace ispan

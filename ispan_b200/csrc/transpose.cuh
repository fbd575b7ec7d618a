// transpose.cuh -- the reverse CSR built on the device from the forward one.
//
// The reference loads both directions from its own files (fw_beg/fw_csr and
// bw_beg/bw_csr, src/graph.cpp:2-92), and the run needs both.  A caller that
// gives only the forward CSR (bw_beg and bw_adj both NULL) gets the reverse
// built here, in HBM, instead of shipping a second copy of the graph over
// PCIe: the in-degrees are counted while the forward adjacency is still
// arriving (one pass per copied chunk), scanned into the reverse offsets, and
// every edge u -> w is then placed in w's list -- by a stable radix sort of
// (w, u) pairs where its scratch fits (lists in increasing source order), else
// by atomics on the offsets themselves: counts at X[w], the inclusive scan
// turns them into the end of each list, and each placement decrements X[w],
// so that once every edge is placed X[w] is the start of w's list (no cursor
// array; lists in no particular order -- the stages never depend on
// adjacency order).
//
// These passes read every forward offset and id, so they also check them
// (offsets from 0 to E, never falling; ids in [0, V)) and raise *bad
// otherwise: the reverse built from a good forward CSR is good by
// construction, and the separate input check (k_validate) is not needed.
// Malformed input must not make them touch memory outside the arrays: ids
// outside [0, V) are skipped, a vertex whose offsets are not
// 0 <= beg <= end <= E places nothing, and a placement outside [0, E) is
// dropped; the run is then refused.
#pragma once
#include "common.cuh"

namespace ispan {

template <typename OffT>
__device__ __forceinline__ void rev_bump(OffT *X, int32_t w, int64_t V, bool &bad) {
    if ((uint64_t)(int64_t)w >= (uint64_t)V) {
        bad = true;
        return;
    }
    if (sizeof(OffT) == 8) atomicAdd(reinterpret_cast<unsigned long long *>(X + w), 1ull);
    else atomicAdd(reinterpret_cast<int *>(X + w), 1);
}

// the offsets of source u, checked: [a, b) with 0 <= a <= b <= E, the first
// offset 0 and the last E; otherwise an empty range and false
template <typename OffT>
__device__ __forceinline__ bool rev_range(const OffT *fb, int64_t u, int64_t V, int64_t E, int64_t &a, int64_t &b) {
    a = (int64_t)fb[u];
    b = (int64_t)fb[u + 1];
    const bool ok = 0 <= a && a <= b && b <= E && (u != 0 || a == 0) && (u != V - 1 || b == E);
    if (!ok) a = b = 0;
    return ok;
}

// The second way to the reverse lists, used where its scratch fits: a copy
// of the forward ids as keys, each edge's source as its value, and a stable
// radix sort of the pairs by key -- the sorted values are the reverse lists,
// each in increasing source order, and no edge needs a returning atomic
// (the placement's atomics run at a third of the count's rate, and at far
// less once the offsets exceed L2).  This fills the values: vals[e] = u for
// the edges e of every source u.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_rev_sources(const OffT *fb, int64_t V, int64_t E, int32_t *vals,
                                                        int *bad) {
    const int lane = lane_id();
    const int64_t gw = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kBlock) >> 5;
    bool bd = false;
    for (int64_t base = gw * 32; base < V; base += nw * 32) {
        const int64_t u = base + lane;
        int64_t a = 0, b = 0;
        if (u < V) bd |= !rev_range(fb, u, V, E, a, b);
        const bool big = b - a >= 32;
        if (!big)
            for (int64_t e = a; e < b; ++e) vals[e] = (int32_t)u;
        for (unsigned m = __ballot_sync(kFull, big); m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            const int64_t s0 = __shfl_sync(kFull, a, src), s1 = __shfl_sync(kFull, b, src);
            for (int64_t e = s0 + lane; e < s1; e += 32) vals[e] = (int32_t)(base + src);
        }
    }
    if (__syncthreads_or(bd) && threadIdx.x == 0) atomicExch(bad, 1);
}

// The sort runs chunk by chunk while the next chunk is still being copied:
// chunk k's (id, source) pairs are sorted on their own (stable), and after
// the last chunk each chunk's runs are placed.  Edges to w from chunk k go
// after those from chunks 0..k-1 (lists stay in increasing source order:
// chunks are in edge order, edges in source order); their offset inside w's
// list is the running in-degree count before chunk k, snapshotted after each
// chunk's count (k_rev_snap), and their offset inside chunk k's sorted run is
// the exclusive scan of chunk k's own counts (k_rev_diff, then a scan).

// snap[w] = the running in-degree count of w (cnt[w] as int32)
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_rev_snap(const OffT *cnt, int64_t V, int32_t *snap) {
    for (int64_t w = (int64_t)blockIdx.x * kBlock + threadIdx.x; w < V; w += (int64_t)gridDim.x * kBlock)
        snap[w] = (int32_t)cnt[w];
}

// d[w] = chunk k's own count of w: snapshot after it minus snapshot before it
__global__ void __launch_bounds__(kBlock) k_rev_diff(const int32_t *after, const int32_t *before, int64_t V,
                                                     int32_t *d) {
    for (int64_t w = (int64_t)blockIdx.x * kBlock + threadIdx.x; w < V; w += (int64_t)gridDim.x * kBlock)
        d[w] = after[w] - (before ? before[w] : 0);
}

// place chunk k's sorted pairs (keys[i], vals[i]), i < n: the pair is the
// (i - run[w])-th of the chunk's edges to w, which follow the before[w]
// edges to w of the earlier chunks in w's list starting at X[w].  A slot
// outside w's list (only on malformed input) is dropped.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_rev_runs(const int32_t *keys, const int32_t *vals, int64_t n,
                                                     const OffT *X, const int32_t *before, const int32_t *run,
                                                     int64_t V, int32_t *ba) {
    for (int64_t i = (int64_t)blockIdx.x * kBlock + threadIdx.x; i < n; i += (int64_t)gridDim.x * kBlock) {
        const int32_t w = keys[i];
        if ((uint64_t)(int64_t)w >= (uint64_t)V) continue;
        const int64_t pos = (int64_t)X[w] + (before ? before[w] : 0) + (i - run[w]);
        if (pos >= (int64_t)X[w] && pos < (int64_t)X[w + 1]) ba[pos] = vals[i];
    }
}

// in-degree counts X[w] += 1 for the edges adj[e0, e1); where adj + e0 is
// 16-byte aligned the body is read as int4 (each id read once, streamed)
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_rev_count(const int32_t *adj, int64_t e0, int64_t e1, int64_t V,
                                                      OffT *X, int *bad) {
    const int64_t gt = (int64_t)blockIdx.x * kBlock + threadIdx.x, nt = (int64_t)gridDim.x * kBlock;
    const int64_t nq = ((uintptr_t)(adj + e0) & 15) ? 0 : (e1 - e0) >> 2;
    const int4 *q = reinterpret_cast<const int4 *>(adj + e0);
    bool b = false;
    for (int64_t i = gt; i < nq; i += nt) {
        const int4 w = __ldcs(q + i);
        rev_bump(X, w.x, V, b);
        rev_bump(X, w.y, V, b);
        rev_bump(X, w.z, V, b);
        rev_bump(X, w.w, V, b);
    }
    for (int64_t e = e0 + (nq << 2) + gt; e < e1; e += nt) rev_bump(X, __ldcs(adj + e), V, b);
    if (__syncthreads_or(b) && threadIdx.x == 0) atomicExch(bad, 1);
}

template <typename OffT>
__device__ __forceinline__ int64_t rev_claim(OffT *X, int32_t w, int64_t V) {
    if ((uint64_t)(int64_t)w >= (uint64_t)V) return -1;
    if (sizeof(OffT) == 8) return (int64_t)atomicAdd(reinterpret_cast<unsigned long long *>(X + w), ~0ull) - 1;
    return (int64_t)atomicAdd(reinterpret_cast<int *>(X + w), -1) - 1;
}

// place the edges fa[e0, e1), e0 + k * stride, of source u: four ids, then
// their four slot claims, then the four stores, so that four returning
// atomics are in flight per thread
template <typename OffT>
__device__ __forceinline__ void rev_place(OffT *X, int32_t *ba, const int32_t *fa, int64_t e0, int64_t e1,
                                          int stride, int32_t u, int64_t V, int64_t E) {
    for (int64_t e = e0; e < e1; e += 4 * stride) {
        int32_t w[4];
        int64_t pos[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) w[q] = e + q * stride < e1 ? __ldcs(fa + e + q * stride) : -1;
#pragma unroll
        for (int q = 0; q < 4; ++q) pos[q] = rev_claim(X, w[q], V);
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (pos[q] >= 0 && pos[q] < E) ba[pos[q]] = u;
    }
}

// place every edge u -> w at the next free slot from the end of w's list.  A
// warp takes 32 consecutive vertices: lists shorter than 32 edges are walked
// by their own lane, longer ones by the whole warp in turn (coalesced reads).
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_rev_fill(const OffT *fb, const int32_t *fa, int64_t V, int64_t E, OffT *X,
                                                     int32_t *ba, int *bad) {
    if (blockIdx.x == 0 && threadIdx.x == 0) X[V] = (OffT)E;
    const int lane = lane_id();
    const int64_t gw = ((int64_t)blockIdx.x * kBlock + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kBlock) >> 5;
    bool bd = false;
    for (int64_t base = gw * 32; base < V; base += nw * 32) {
        const int64_t u = base + lane;
        int64_t a = 0, b = 0;
        if (u < V) bd |= !rev_range(fb, u, V, E, a, b);
        const bool big = b - a >= 32;
        if (!big) rev_place(X, ba, fa, a, b, 1, (int32_t)u, V, E);
        for (unsigned m = __ballot_sync(kFull, big); m; m &= m - 1) {
            const int src = __ffs(m) - 1;
            const int64_t s0 = __shfl_sync(kFull, a, src), s1 = __shfl_sync(kFull, b, src);
            rev_place(X, ba, fa, s0 + lane, s1, 32, (int32_t)(base + src), V, E);
        }
    }
    if (__syncthreads_or(bd) && threadIdx.x == 0) atomicExch(bad, 1);
}

}  // namespace ispan

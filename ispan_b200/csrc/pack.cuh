// pack.cuh -- packing many independent graphs into one disjoint union and
// unpacking its labels (ispan_scc_run_graphs and the server).
//
// Graph i of a batch keeps its own CSR (offsets of 4 or 8 bytes, local ids);
// the union has int64 offsets and global ids: graph i's vertices start at
// vbase[i] and its edges at ebase[i].  The reference has no counterpart (it
// runs one graph per process, src/scc_main.cpp:41-47).
//
// The pack kernels also check every input graph, so the union is well formed
// by construction: offsets start at 0, never decrease and end at E; every
// adjacency id lies in [0, V).  A violation sets *err and the batch is
// rejected before any stage kernel runs.
#pragma once
#include <cstdint>

namespace ispan {

struct PackDesc {
    const void *fw_beg, *bw_beg;      // offsets, ob bytes each (device memory)
    const int32_t *fw_adj, *bw_adj;   // local ids (device memory; may alias the union)
    int64_t V, E, vbase, ebase;
    int32_t ob, pad;
};

constexpr int kPackTile = 8192;   // elements per CTA tile
constexpr int kPackThreads = 256;

// largest s in [lo, hi] with b[s] <= i (b non-decreasing, b[lo] <= i)
__device__ __forceinline__ int pack_seg(const int64_t *b, int lo, int hi, int64_t i) {
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(b + mid) <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int64_t pack_off(const void *p, int64_t j, int ob) {
    return ob == 4 ? (int64_t)__ldg(reinterpret_cast<const int32_t *>(p) + j)
                   : __ldg(reinterpret_cast<const long long *>(p) + j);
}

// Union offsets: slot i < Vt takes graph s's offset of its local vertex plus
// ebase[s]; slot Vt is the edge total.  b = vbase[0..n].
__global__ void __launch_bounds__(kPackThreads) k_pack_offsets(const PackDesc *__restrict__ d, int n,
                                                               const int64_t *__restrict__ b, int64_t Vt,
                                                               int64_t Et, int64_t *__restrict__ fwb,
                                                               int64_t *__restrict__ bwb, int *err) {
    __shared__ int s_lo, s_hi;
    for (int64_t t0 = (int64_t)blockIdx.x * kPackTile; t0 <= Vt; t0 += (int64_t)gridDim.x * kPackTile) {
        const int64_t t1 = min(Vt, t0 + kPackTile);  // slots [t0, t1) plus Vt itself below
        if (threadIdx.x == 0 && t0 < t1) {
            s_lo = pack_seg(b, 0, n - 1, t0);
            s_hi = pack_seg(b, 0, n - 1, t1 - 1);
        }
        __syncthreads();
        const int lo = s_lo, hi = s_hi;
        for (int64_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
            const int s = lo == hi ? lo : pack_seg(b, lo, hi, i);
            const PackDesc D = d[s];
            const int64_t j = i - D.vbase;
            const int64_t f0 = pack_off(D.fw_beg, j, D.ob), f1 = pack_off(D.fw_beg, j + 1, D.ob);
            const int64_t b0 = pack_off(D.bw_beg, j, D.ob), b1 = pack_off(D.bw_beg, j + 1, D.ob);
            bool ok = f0 <= f1 && b0 <= b1 && f1 <= D.E && b1 <= D.E;
            if (j == 0) ok = ok && f0 == 0 && b0 == 0;
            if (j + 1 == D.V) ok = ok && f1 == D.E && b1 == D.E;
            if (!ok) atomicCAS(err, 0, 1);
            fwb[i] = D.ebase + f0;
            bwb[i] = D.ebase + b0;
        }
        if (t0 <= Vt && Vt < t0 + kPackTile && threadIdx.x == 0) {
            fwb[Vt] = Et;
            bwb[Vt] = Et;
        }
        __syncthreads();
    }
}

// Union adjacency: edge slot e of graph s takes its local id plus vbase[s].
// In place when the descriptor's adjacency already is the union slice (host
// input copied there): each element is read and written by the same thread.
// b = ebase[0..n].
__global__ void __launch_bounds__(kPackThreads) k_pack_adj(const PackDesc *__restrict__ d, int n,
                                                           const int64_t *__restrict__ b, int64_t Et,
                                                           int32_t *fwa, int32_t *bwa, int *err) {
    __shared__ int s_lo, s_hi;
    for (int64_t t0 = (int64_t)blockIdx.x * kPackTile; t0 < Et; t0 += (int64_t)gridDim.x * kPackTile) {
        const int64_t t1 = min(Et, t0 + kPackTile);
        if (threadIdx.x == 0) {
            s_lo = pack_seg(b, 0, n - 1, t0);
            s_hi = pack_seg(b, 0, n - 1, t1 - 1);
        }
        __syncthreads();
        const int lo = s_lo, hi = s_hi;
        for (int64_t e = t0 + threadIdx.x; e < t1; e += blockDim.x) {
            const int s = lo == hi ? lo : pack_seg(b, lo, hi, e);
            const int64_t j = e - __ldg(&d[s].ebase);
            const int64_t V = __ldg(&d[s].V), vb = __ldg(&d[s].vbase);
            const int32_t x = d[s].fw_adj[j], y = d[s].bw_adj[j];
            if ((uint64_t)(int64_t)x >= (uint64_t)V || (uint64_t)(int64_t)y >= (uint64_t)V) atomicCAS(err, 0, 2);
            fwa[e] = (int32_t)(x + vb);
            bwa[e] = (int32_t)(y + vb);
        }
        __syncthreads();
    }
}

// Union labels (global min ids) back to each graph's local ids, in place.
__global__ void __launch_bounds__(kPackThreads) k_unpack_labels(int32_t *label, int n,
                                                                const int64_t *__restrict__ b, int64_t Vt) {
    __shared__ int s_lo, s_hi;
    for (int64_t t0 = (int64_t)blockIdx.x * kPackTile; t0 < Vt; t0 += (int64_t)gridDim.x * kPackTile) {
        const int64_t t1 = min(Vt, t0 + kPackTile);
        if (threadIdx.x == 0) {
            s_lo = pack_seg(b, 0, n - 1, t0);
            s_hi = pack_seg(b, 0, n - 1, t1 - 1);
        }
        __syncthreads();
        const int lo = s_lo, hi = s_hi;
        for (int64_t i = t0 + threadIdx.x; i < t1; i += blockDim.x) {
            const int s = lo == hi ? lo : pack_seg(b, lo, hi, i);
            label[i] -= (int32_t)__ldg(b + s);
        }
        __syncthreads();
    }
}

}  // namespace ispan

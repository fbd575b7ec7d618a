// condense.cu -- the condensation of a graph given its SCC labels: the DAG
// whose vertices are the SCCs (named by their canonical labels, the minimum
// vertex id) and whose edges are the distinct label pairs of the graph's
// edges that cross two SCCs (ispan_condense in include/ispan_b200.h).
//
// The reference stops at class counts (src/load_print.cpp:24-60); this is
// the step after the path that a caller of an SCC detector usually needs
// next (topological order of components, reachability summaries).
//
// One pass over the forward CSR emits the crossing pairs as 64-bit keys
// (source label << 32 | target label) with one warp-aggregated reservation
// per warp; a radix sort and a unique pass leave them sorted and distinct.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "../../include/ispan_b200.h"

namespace {

constexpr int kThreads = 256;

template <typename OffT>
__global__ void __launch_bounds__(kThreads) k_cross_pairs(const OffT *__restrict__ beg, const int32_t *__restrict__ adj,
                                                          const int32_t *__restrict__ label, int64_t V,
                                                          unsigned long long *out, unsigned long long *count,
                                                          int64_t cap) {
    // warp per vertex run: lanes stride the vertex's edges
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * kThreads) >> 5;
    for (int64_t u = warp; u < V; u += nwarps) {
        const int64_t e0 = (int64_t)beg[u], e1 = (int64_t)beg[u + 1];
        const uint32_t lu = (uint32_t)__ldg(label + u);
        for (int64_t e = e0; e - lane < e1; e += 32) {
            bool cross = false;
            unsigned long long key = 0;
            if (e + lane < e1) {
                const int32_t w = __ldg(adj + e + lane);
                if ((uint64_t)(int64_t)w < (uint64_t)V) {  // ids outside [0, V) are skipped
                    const uint32_t lw = (uint32_t)__ldg(label + w);
                    cross = lw != lu;
                    key = ((unsigned long long)lu << 32) | lw;
                }
            }
            const unsigned m = __ballot_sync(0xffffffffu, cross);
            if (!m) continue;
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(count, (unsigned long long)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (cross) {
                const unsigned long long slot = base + __popc(m & ((1u << lane) - 1u));
                if ((int64_t)slot < cap) out[slot] = key;
            }
        }
    }
}

#define CKC(x)                                                                                 \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            fprintf(stderr, "ispan_condense: %s failed: %s\n", #x, cudaGetErrorString(e_));  \
            rc = e_ == cudaErrorMemoryAllocation ? ISPAN_ERR_NOMEM : ISPAN_ERR_CUDA;          \
            goto done;                                                                         \
        }                                                                                      \
    } while (0)

}  // namespace

extern "C" int ispan_condense(const ispan_csr *g, const int32_t *labels, uint64_t *pairs_out, int64_t cap,
                              int64_t *n_pairs, void *stream) {
    if (!g || !labels || !n_pairs || !g->on_device || (g->offset_bytes != 4 && g->offset_bytes != 8) || g->V < 0 ||
        g->E < 0 || cap < 0 || (cap > 0 && !pairs_out))
        return ISPAN_ERR_ARG;
    *n_pairs = 0;
    if (g->V == 0 || g->E == 0) return ISPAN_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int rc = ISPAN_OK;
    unsigned long long *keys = nullptr, *sorted = nullptr, *cnt = nullptr, h_cnt = 0;
    int64_t *n_uniq = nullptr, h_uniq = 0;
    void *tmp = nullptr;
    size_t t1 = 0, t2 = 0;
    int64_t n = 0;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = nsm * 8;
    // first pass counts the crossing edges (cap 0), the second writes them
    CKC(cudaMalloc(&cnt, sizeof(unsigned long long)));
    CKC(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
    if (g->offset_bytes == 4)
        k_cross_pairs<int32_t><<<grid, kThreads, 0, s>>>((const int32_t *)g->fw_beg, g->fw_adj, labels, g->V, nullptr,
                                                         cnt, 0);
    else
        k_cross_pairs<int64_t><<<grid, kThreads, 0, s>>>((const int64_t *)g->fw_beg, g->fw_adj, labels, g->V, nullptr,
                                                         cnt, 0);
    CKC(cudaGetLastError());
    CKC(cudaMemcpyAsync(&h_cnt, cnt, sizeof h_cnt, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    n = (int64_t)h_cnt;
    if (n == 0) goto done;
    CKC(cudaMalloc(&keys, n * sizeof(unsigned long long)));
    CKC(cudaMalloc(&sorted, n * sizeof(unsigned long long)));
    CKC(cudaMalloc(&n_uniq, sizeof(int64_t)));
    CKC(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
    if (g->offset_bytes == 4)
        k_cross_pairs<int32_t><<<grid, kThreads, 0, s>>>((const int32_t *)g->fw_beg, g->fw_adj, labels, g->V, keys,
                                                         cnt, n);
    else
        k_cross_pairs<int64_t><<<grid, kThreads, 0, s>>>((const int64_t *)g->fw_beg, g->fw_adj, labels, g->V, keys,
                                                         cnt, n);
    CKC(cudaGetLastError());
    CKC(cub::DeviceRadixSort::SortKeys(nullptr, t1, keys, sorted, n, 0, 64, s));
    CKC(cub::DeviceSelect::Unique(nullptr, t2, sorted, keys, n_uniq, n, s));
    CKC(cudaMalloc(&tmp, std::max(t1, t2) + 256));
    CKC(cub::DeviceRadixSort::SortKeys(tmp, t1, keys, sorted, n, 0, 64, s));
    CKC(cub::DeviceSelect::Unique(tmp, t2, sorted, keys, n_uniq, n, s));
    CKC(cudaMemcpyAsync(&h_uniq, n_uniq, sizeof h_uniq, cudaMemcpyDeviceToHost, s));
    CKC(cudaStreamSynchronize(s));
    *n_pairs = h_uniq;
    if (cap > 0)
        CKC(cudaMemcpyAsync(pairs_out, keys, (size_t)std::min(cap, h_uniq) * sizeof(uint64_t), cudaMemcpyDefault, s));
    CKC(cudaStreamSynchronize(s));
done:
    cudaFree(keys);
    cudaFree(sorted);
    cudaFree(cnt);
    cudaFree(n_uniq);
    cudaFree(tmp);
    return rc;
}

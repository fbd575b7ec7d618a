// shard.cu -- one rank's step of a reachability search over a graph whose
// rows are split across GPUs (ispan_shard_expand in include/ispan_b200.h).
//
// The reference's distributed variant partitions the vertex range across MPI
// ranks and, per BFS level, merges the ranks' frontier state with a MAX
// all-reduce over a byte per vertex (src_mpi/fw_bw.h:193, :309) or a bitwise
// OR over a bitmap (:382-442).  Here each rank owns the CSR rows of a vertex
// range [v0, v1) (global ids in the adjacency); a level is this kernel --
// every owned frontier vertex marks its allowed, unvisited neighbours in a
// full-length next-frontier byte map -- followed by a MAX all-reduce of that
// map over NCCL (ispan_b200/sharded.py), after which every rank holds the
// same next frontier.  Byte maps, not bitmaps: plain stores need no atomics
// and NCCL reduces bytes with MAX.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ispan_b200.h"

namespace {

template <typename OffT>
__global__ void k_shard_expand(const OffT *__restrict__ beg, const int32_t *__restrict__ adj, int64_t v0, int64_t nv,
                               int64_t V, const uint8_t *__restrict__ frontier, const uint8_t *__restrict__ visited,
                               const uint8_t *__restrict__ allowed, uint8_t *next) {
    // a warp per owned vertex: lanes stride its edges
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t i = warp; i < nv; i += nwarps) {
        if (!frontier[v0 + i]) continue;
        const int64_t e0 = (int64_t)beg[i], e1 = (int64_t)beg[i + 1];
        for (int64_t e = e0 + lane; e < e1; e += 32) {
            const int32_t w = adj[e];
            if ((uint64_t)(int64_t)w >= (uint64_t)V) continue;  // ids outside [0, V) are ignored
            if (visited[w] || (allowed && !allowed[w])) continue;
            next[w] = 1;  // idempotent: no atomic needed
        }
    }
}

}  // namespace

extern "C" int ispan_shard_expand(const ispan_csr *rows, int64_t v0, int64_t V, const uint8_t *frontier,
                                  const uint8_t *visited, const uint8_t *allowed, uint8_t *next, void *stream) {
    if (!rows || !rows->on_device || (rows->offset_bytes != 4 && rows->offset_bytes != 8) || rows->V < 0 ||
        v0 < 0 || V < 0 || v0 + rows->V > V || !frontier || !visited || !next)
        return ISPAN_ERR_ARG;
    if (rows->V == 0 || rows->E == 0) return ISPAN_OK;
    if (!rows->fw_beg || !rows->fw_adj) return ISPAN_ERR_ARG;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = 256, grid = nsm * 8;
    if (rows->offset_bytes == 4)
        k_shard_expand<int32_t><<<grid, threads, 0, s>>>((const int32_t *)rows->fw_beg, rows->fw_adj, v0, rows->V, V,
                                                          frontier, visited, allowed, next);
    else
        k_shard_expand<int64_t><<<grid, threads, 0, s>>>((const int64_t *)rows->fw_beg, rows->fw_adj, v0, rows->V, V,
                                                          frontier, visited, allowed, next);
    return cudaGetLastError() == cudaSuccess ? ISPAN_OK : ISPAN_ERR_CUDA;
}

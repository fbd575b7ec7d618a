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
//
// The queue form (ispan_shard_expand_queue + ispan_shard_collect) is what
// ispan_b200/sharded.py runs: each rank expands only its owned frontier
// queue, the next-frontier byte maps are merged by a reduce-scatter (MAX),
// so each rank receives just its owned slice, the owner filters it against
// its visited bits and queues the new vertices, and the visited bitmap is
// replicated by an all-gather of the owned words (packed bits).  Per level
// that moves V bytes into the reduce-scatter and V/8 bytes of all-gather,
// against V bytes of all-reduce (which moves twice the data) in the byte-map
// form, and the work is proportional to the frontier's edges.
#include <cuda_runtime.h>

#include <algorithm>
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

// Queue form of a level: warps take the owned frontier vertices from a queue
// (count read on the device) instead of testing every owned vertex's byte;
// visited and restriction state are replicated bitmaps (V bits).
template <typename OffT>
__global__ void k_shard_expand_queue(const OffT *__restrict__ beg, const int32_t *__restrict__ adj, int64_t v0,
                                     int64_t nv, int64_t V, const int32_t *__restrict__ queue,
                                     const int64_t *__restrict__ qn, const uint32_t *__restrict__ visited,
                                     const uint32_t *__restrict__ allowed, uint8_t *next) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t n = *qn;
    for (int64_t k = warp; k < n; k += nwarps) {
        const int64_t i = (int64_t)queue[k] - v0;
        if ((uint64_t)i >= (uint64_t)nv) continue;  // not an owned vertex
        const int64_t e0 = (int64_t)beg[i], e1 = (int64_t)beg[i + 1];
        for (int64_t e = e0 + lane; e < e1; e += 32) {
            const int32_t w = adj[e];
            if ((uint64_t)(int64_t)w >= (uint64_t)V) continue;  // ids outside [0, V) are ignored
            const uint32_t b = 1u << (w & 31);
            if ((visited[w >> 5] & b) || (allowed && !(allowed[w >> 5] & b))) continue;
            next[w] = 1;  // idempotent: no atomic needed
        }
    }
}

// The owner's half of a level: owned vertices set in the merged next map
// and not yet visited become visited and form the next owned queue.  One
// thread per owned word (v0 is a multiple of 32).
__global__ void k_shard_collect(int64_t v0, int64_t nv, const uint8_t *__restrict__ mine, uint32_t *visited,
                                int32_t *queue, unsigned long long *qn) {
    const int lane = threadIdx.x & 31;
    const int64_t nw = (nv + 31) / 32;
    for (int64_t wi = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; wi - lane < nw;
         wi += (int64_t)gridDim.x * blockDim.x) {
        uint32_t m = 0;
        if (wi < nw) {
            for (int j = 0; j < 32; ++j) {
                const int64_t i = wi * 32 + j;
                if (i < nv && mine[i]) m |= 1u << j;
            }
            m &= ~visited[(v0 >> 5) + wi];
            visited[(v0 >> 5) + wi] |= m;
        }
        // warp-aggregated append of the word's new vertices, in id order
        const int c = __popc(m);
        int incl = c;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int tot = __shfl_sync(0xffffffffu, incl, 31);
        unsigned long long base = 0;
        if (lane == 31 && tot) base = atomicAdd(qn, (unsigned long long)tot);
        base = __shfl_sync(0xffffffffu, base, 31);
        long long at = (long long)base + incl - c;
        for (; m; m &= m - 1) queue[at++] = (int32_t)(v0 + wi * 32 + __ffs(m) - 1);
    }
}

}  // namespace

extern "C" int ispan_shard_expand_queue(const ispan_csr *rows, int64_t v0, int64_t V, const int32_t *queue,
                                        const int64_t *queue_count, const uint32_t *visited,
                                        const uint32_t *allowed, uint8_t *next, void *stream) {
    if (!rows || !rows->on_device || (rows->offset_bytes != 4 && rows->offset_bytes != 8) || rows->V < 0 ||
        v0 < 0 || V < 0 || v0 + rows->V > V || !queue || !queue_count || !visited || !next)
        return ISPAN_ERR_ARG;
    if (rows->V == 0 || rows->E == 0) return ISPAN_OK;
    if (!rows->fw_beg || !rows->fw_adj) return ISPAN_ERR_ARG;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = 256, grid = nsm * 8;
    if (rows->offset_bytes == 4)
        k_shard_expand_queue<int32_t><<<grid, threads, 0, s>>>((const int32_t *)rows->fw_beg, rows->fw_adj, v0,
                                                                rows->V, V, queue, queue_count, visited, allowed,
                                                                next);
    else
        k_shard_expand_queue<int64_t><<<grid, threads, 0, s>>>((const int64_t *)rows->fw_beg, rows->fw_adj, v0,
                                                                rows->V, V, queue, queue_count, visited, allowed,
                                                                next);
    return cudaGetLastError() == cudaSuccess ? ISPAN_OK : ISPAN_ERR_CUDA;
}

extern "C" int ispan_shard_collect(int64_t v0, int64_t n_own, const uint8_t *mine, uint32_t *visited,
                                   int32_t *queue, int64_t *queue_count, void *stream) {
    if (v0 < 0 || (v0 & 31) || n_own < 0 || !mine || !visited || !queue || !queue_count) return ISPAN_ERR_ARG;
    if (n_own == 0) return ISPAN_OK;
    const int64_t nw = (n_own + 31) / 32;
    const int grid = (int)std::min<int64_t>((nw + 255) / 256, 4096);
    k_shard_collect<<<grid, 256, 0, (cudaStream_t)stream>>>(v0, n_own, mine, visited, queue,
                                                             (unsigned long long *)queue_count);
    return cudaGetLastError() == cudaSuccess ? ISPAN_OK : ISPAN_ERR_CUDA;
}

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

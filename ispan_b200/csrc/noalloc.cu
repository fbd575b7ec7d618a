// noalloc.cu -- SCC labels of one small device-resident graph without any
// device allocation (ispan_scc_small_noalloc in include/ispan_b200.h).
//
// Some callers cannot call cudaMalloc: code that runs under another
// framework's memory manager (which owns the device memory and does not
// allow private allocations), latency-critical paths where cudaMalloc's
// implicit synchronisation is not acceptable, and code that issues work
// while a stream is being captured, where allocation calls are not
// permitted.  For them this entry point keeps its scratch in a file-scope
// device array of fixed size, so a call only launches one kernel.
//
// The kernel is the serial Tarjan of k_local_scc (stages.cuh) run by one
// thread of one CTA over the whole graph, with its per-vertex stacks in the
// static scratch instead of shared memory; the other threads initialise the
// scratch.  Labels are the minimum vertex id of each SCC, as from
// ispan_scc_run.  The kernel first checks the graph (offsets monotone from 0
// to E, ids in [0, V)) and answers a malformed one with -1 labels, so a bad
// id can never index past the scratch.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/ispan_b200.h"

namespace {

constexpr int64_t kMaxV = ISPAN_NOALLOC_MAX_V;
// per vertex: index, lowlink, stack entry, call-stack vertex (int32 each),
// call-stack edge cursor (int64), on-stack flag (byte), padded to 32 bytes
constexpr size_t kBytesPerVertex = 32;
constexpr size_t kScratchBytes = (size_t)kMaxV * kBytesPerVertex;  // 2 MiB

// Shared by every call on a device; holds the previous call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Host-side addresses of g_noalloc_scratch, one per device (the symbol name
// in host code is not a device address).
constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_setup_mu;

template <typename OffT>
__global__ void __launch_bounds__(256) k_scc_small_static(const OffT *__restrict__ fw_beg,
                                                          const int32_t *__restrict__ fw_adj, int64_t V, int64_t E,
                                                          int32_t *__restrict__ labels, unsigned char *scratch) {
    int32_t *idx = reinterpret_cast<int32_t *>(scratch);
    int32_t *low = idx + kMaxV;
    int32_t *stk = low + kMaxV;
    int32_t *csv = stk + kMaxV;
    int64_t *cse = reinterpret_cast<int64_t *>(csv + kMaxV);
    unsigned char *onst = reinterpret_cast<unsigned char *>(cse + kMaxV);
    // Input check before any index taken from the graph is used: offsets
    // monotone from 0 to E, every adjacency id in [0, V).  These loops read
    // only fw_beg[0..V] and fw_adj[0..E), the arrays the caller declared.  A
    // malformed graph gets -1 in every label and nothing else is touched (the
    // Tarjan below indexes the scratch with adjacency ids).
    int bad = 0;
    for (int64_t v = threadIdx.x; v <= V; v += blockDim.x) {
        const int64_t a = (int64_t)fw_beg[v];
        if ((v == 0 && a != 0) || (v == V && a != E) || (v < V && (int64_t)fw_beg[v + 1] < a)) bad = 1;
    }
    for (int64_t e = threadIdx.x; e < E; e += blockDim.x) {
        const int32_t w = fw_adj[e];
        if (w < 0 || w >= V) bad = 1;
    }
    if (__syncthreads_or(bad)) {
        for (int64_t v = threadIdx.x; v < V; v += blockDim.x) labels[v] = -1;
        return;
    }
    // the scratch keeps the last call's contents: reset what must start clear
    for (int64_t v = threadIdx.x; v < V; v += blockDim.x) {
        idx[v] = -1;
        onst[v] = 0;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    int32_t counter = 0, sp = 0;
    for (int64_t s0 = 0; s0 < V; ++s0) {
        if (idx[s0] != -1) continue;
        int64_t cp = 0;
        csv[0] = (int32_t)s0;
        cse[0] = (int64_t)fw_beg[s0];
        cp = 1;
        idx[s0] = low[s0] = counter++;
        stk[sp++] = (int32_t)s0;
        onst[s0] = 1;
        while (cp > 0) {
            const int32_t v = csv[cp - 1];
            int64_t e = cse[cp - 1];
            const int64_t end = (int64_t)fw_beg[v + 1];
            bool down = false;
            for (; e < end; ++e) {
                const int32_t w = fw_adj[e];
                if (idx[w] == -1) {
                    cse[cp - 1] = e + 1;
                    idx[w] = low[w] = counter++;
                    stk[sp++] = w;
                    onst[w] = 1;
                    csv[cp] = w;
                    cse[cp] = (int64_t)fw_beg[w];
                    ++cp;
                    down = true;
                    break;
                } else if (onst[w] && idx[w] < low[v]) {
                    low[v] = idx[w];
                }
            }
            if (down) continue;
            if (low[v] == idx[v]) {
                int32_t mn = 0x7fffffff;
                int32_t k = sp;
                do {
                    --k;
                    mn = min(mn, stk[k]);
                } while (stk[k] != v);
                while (sp > k) {
                    const int32_t w = stk[--sp];
                    onst[w] = 0;
                    labels[w] = mn;
                }
            }
            --cp;
            if (cp > 0) {
                const int32_t p = csv[cp - 1];
                if (low[v] < low[p]) low[p] = low[v];
            }
        }
    }
}

}  // namespace

extern "C" int ispan_scc_small_noalloc(const ispan_csr *g, int32_t *labels_out, void *stream) {
    if (!g || !g->on_device || (g->offset_bytes != 4 && g->offset_bytes != 8) || g->V < 0 || g->E < 0)
        return ISPAN_ERR_ARG;
    if (g->V > kMaxV) {
        fprintf(stderr, "ispan_scc_small_noalloc: %lld vertices exceed the static scratch limit of %lld\n",
                (long long)g->V, (long long)kMaxV);
        return ISPAN_ERR_CAPACITY;
    }
    if (g->V == 0) return ISPAN_OK;
    if (!g->fw_beg || !labels_out || (g->E > 0 && !g->fw_adj)) return ISPAN_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return ISPAN_ERR_CUDA;
    void *scratch = nullptr;
    {
        // first call on a device: resolve the scratch array's device address
        // with that device current (this is the only set-up; make the first
        // call before any stream capture)
        std::lock_guard<std::mutex> lock(g_setup_mu);
        if (!g_scratch_addr[dev]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                fprintf(stderr, "ispan_scc_small_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
                return ISPAN_ERR_CUDA;
            }
            g_scratch_addr[dev] = p;
        }
        scratch = g_scratch_addr[dev];
    }
    // an error left pending by earlier work on this thread is reported, not
    // cleared, and no launch is made
    if (cudaPeekAtLastError() != cudaSuccess) return ISPAN_ERR_CUDA;
    cudaStream_t s = (cudaStream_t)stream;
    if (g->offset_bytes == 4)
        k_scc_small_static<int32_t><<<1, 256, 0, s>>>((const int32_t *)g->fw_beg, g->fw_adj, g->V, g->E,
                                                       labels_out, (unsigned char *)scratch);
    else
        k_scc_small_static<int64_t><<<1, 256, 0, s>>>((const int64_t *)g->fw_beg, g->fw_adj, g->V, g->E,
                                                       labels_out, (unsigned char *)scratch);
    // nothing was pending before the launch, so this is the launch's own status
    return cudaGetLastError() == cudaSuccess ? ISPAN_OK : ISPAN_ERR_CUDA;
}

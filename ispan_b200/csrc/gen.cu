// gen.cu -- seeded synthetic graphs built on the GPU (include/ispan_gen.h).
//
// Every generator is an "edge program": a list of categories, each emitting a
// known number of edges as 64-bit keys (src << 32 | dst) from a counter-based
// hash of (seed, category, item), so the graph depends only on the seed and
// the sizes.  Keys are radix-sorted (CUB), self-loops and duplicates dropped,
// and both CSR directions built from the sorted keys.  Vertex roles are
// assigned to ranks, and ranks are scattered over vertex ids by a seeded
// bijection (a Feistel network with cycle walking, shifted so vertex 0 is
// rank 0), so hubs and classes do not sit at low ids.
//
// These are input builders for tests and benchmarks; they are not part of the
// SCC pipeline and are never timed.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/ispan_gen.h"

struct PlantedInfo;
struct ispan_gen_graph {
    int device = 0;
    int64_t V = 0, E = 0;
    int64_t *fw_beg = nullptr, *bw_beg = nullptr;
    int32_t *fw_adj = nullptr, *bw_adj = nullptr;
    PlantedInfo *planted = nullptr;  // the SCC partition the generator planted (social, web)
};

namespace {

#define GK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            fprintf(stderr, "ispan_gen: %s: %s (%s:%d)\n", #x, cudaGetErrorString(e_), __FILE__, \
                    __LINE__);                                                                  \
            return -3;                                                                          \
        }                                                                                       \
    } while (0)

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    // splitmix64 finaliser
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t rnd(uint64_t seed, uint32_t cat, uint64_t item, uint32_t k) {
    return mix64(seed ^ mix64(((uint64_t)cat << 40) ^ ((uint64_t)k << 56) ^ item));
}
__host__ __device__ __forceinline__ double u01(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

// Seeded bijection on [0, n): 4-round Feistel over 2^(2h) >= n, cycle walking.
struct Perm {
    int64_t n;
    int half;
    uint64_t key;
    int64_t shift;  // perm(0), so that rank(v) = (perm(v) - perm(0)) mod n
    __host__ __device__ uint64_t f(uint64_t x, int r) const { return mix64(x ^ (key + 0x1000193ull * (r + 1))); }
    __host__ __device__ uint64_t fwd1(uint64_t x) const {
        uint64_t m = (1ull << half) - 1, L = x >> half, R = x & m;
        for (int r = 0; r < 4; ++r) {
            uint64_t nl = R;
            R = L ^ (f(R, r) & m);
            L = nl;
        }
        return (L << half) | R;
    }
    __host__ __device__ uint64_t inv1(uint64_t x) const {
        uint64_t m = (1ull << half) - 1, L = x >> half, R = x & m;
        for (int r = 3; r >= 0; --r) {
            uint64_t nr = L;
            L = R ^ (f(L, r) & m);
            R = nr;
        }
        return (L << half) | R;
    }
    __host__ __device__ int64_t fwd(int64_t x) const {
        uint64_t y = fwd1((uint64_t)x);
        while (y >= (uint64_t)n) y = fwd1(y);
        return (int64_t)y;
    }
    __host__ __device__ int64_t inv(int64_t x) const {
        uint64_t y = inv1((uint64_t)x);
        while (y >= (uint64_t)n) y = inv1(y);
        return (int64_t)y;
    }
    // vertex id of a rank
    __host__ __device__ int64_t vertex(int64_t rank) const {
        int64_t p = rank + shift;
        if (p >= n) p -= n;
        return inv(p);
    }
    // rank0: the rank that vertex 0 receives
    static Perm make(int64_t n, uint64_t seed, int64_t rank0 = 0) {
        Perm p;
        p.n = std::max<int64_t>(n, 1);
        int bits = 2;
        while ((1ll << bits) < p.n) ++bits;
        if (bits & 1) ++bits;
        p.half = bits / 2;
        p.key = mix64(seed ^ 0x5eedull);
        p.shift = 0;
        p.shift = (p.fwd(0) - rank0 % p.n + p.n) % p.n;
        return p;
    }
};

// Inverse-CDF sampler of ranks [0, n) with weight (i + i0)^-beta.
struct PowerLaw {
    double i0, beta, A, Bm, inv1mb;
    int64_t n;
    __host__ __device__ int64_t sample(double u) const {
        double x;
        if (fabs(1.0 - beta) < 1e-9) {
            x = exp(log(i0) + u * (log(n + i0) - log(i0))) - i0;
        } else {
            x = pow(A + u * (Bm - A), inv1mb) - i0;
        }
        int64_t r = (int64_t)x;
        return r < 0 ? 0 : (r >= n ? n - 1 : r);
    }
    // expected share of rank 0
    static double top_share(int64_t n, double beta, double i0) {
        if (fabs(1.0 - beta) < 1e-9) return pow(i0, -beta) / (log(n + i0) - log(i0));
        return pow(i0, -beta) * (1.0 - beta) / (pow(n + i0, 1.0 - beta) - pow(i0, 1.0 - beta));
    }
    static PowerLaw make(int64_t n, double beta, double i0) {
        PowerLaw p;
        p.n = std::max<int64_t>(n, 1);
        p.beta = beta;
        p.i0 = i0;
        p.A = pow(i0, 1.0 - beta);
        p.Bm = pow(n + i0, 1.0 - beta);
        p.inv1mb = 1.0 / (1.0 - beta);
        return p;
    }
    // choose i0 so that rank 0 expects `top` of `total` samples
    static PowerLaw fit(int64_t n, double beta, double total, double top) {
        double lo = 1e-3, hi = (double)n;
        for (int it = 0; it < 200; ++it) {
            double mid = sqrt(lo * hi);
            if (top_share(n, beta, mid) * total > top) lo = mid; else hi = mid;
        }
        return make(n, beta, sqrt(lo * hi));
    }
};

// ---------------------------------------------------------------------------
// The SCC partition a generator planted, in rank space: the core [0, n_core)
// is one SCC, the ranks [block_lo, block_lo + bnd.back()) are cut into SCCs
// at the relative boundaries bnd, every other rank is an SCC of its own.  A
// vertex's planted label is the minimum vertex id of its SCC.
}  // namespace

struct PlantedInfo {  // declared with ispan_gen_graph, outside the file's unnamed namespace
    Perm perm;
    int64_t n = 0, n_core = 0, block_lo = 0;
    std::vector<int64_t> bnd;
};

namespace {

__device__ __forceinline__ int64_t planted_group(int64_t r, int64_t n_core, int64_t block_lo, const int64_t *bnd,
                                                 int64_t nb) {
    if (r < n_core) return 0;
    const int64_t x = r - block_lo;
    if (x < 0 || x >= bnd[nb]) return -1;
    int64_t lo = 0, hi = nb - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi + 1) >> 1;
        if (bnd[mid] <= x) lo = mid; else hi = mid - 1;
    }
    return 1 + lo;
}

__global__ void k_planted_min(Perm perm, int64_t n, int64_t n_core, int64_t block_lo, const int64_t *bnd,
                              int64_t nb, int32_t *gmin) {
    // grid-stride with whole warps in every iteration, so lanes of the same
    // group (the core is a third of all ranks) combine before one atomic
    const int lane = threadIdx.x & 31;
    for (int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x - lane; r0 < n;
         r0 += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = r0 + lane;
        const int64_t gi = r < n ? planted_group(r, n_core, block_lo, bnd, nb) : -1;
        const uint32_t v = r < n ? (uint32_t)perm.vertex(r) : 0xffffffffu;
        const unsigned grp = __match_any_sync(0xffffffffu, (unsigned long long)gi);
        const uint32_t mv = __reduce_min_sync(grp, v);
        if (gi >= 0 && lane == __ffs(grp) - 1) atomicMin(gmin + gi, (int32_t)mv);
    }
}

__global__ void k_planted_label(Perm perm, int64_t n, int64_t n_core, int64_t block_lo, const int64_t *bnd,
                                int64_t nb, const int32_t *gmin, int32_t *label) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gi = planted_group(r, n_core, block_lo, bnd, nb);
        const int64_t v = perm.vertex(r);
        label[v] = gi >= 0 ? gmin[gi] : (int32_t)v;
    }
}

// ---------------------------------------------------------------------------
// social-network edge program
enum SocCat : uint32_t {
    S_RING = 1, S_CL, S_SRC0, S_SRCX, S_SNK0, S_SNKX, S_UP, S_DN, S_PAIR, S_TRI, S_TAIL, S_NCAT
};
struct SocProg {
    Perm perm;
    Perm ring;  // order of the Hamiltonian cycle over the core ranks
    uint64_t seed;
    int64_t n_core, n_src, n_snk, n_up, n_dn, n_pair, n_tri, n_tail_v, n_tail;
    int64_t b_src, b_snk, b_up, b_dn, b_pair, b_tri, b_tail;  // rank bases
    PowerLaw pl_out, pl_in, pl_src, pl_snk;
    int64_t cat_begin[S_NCAT + 1];  // item ranges (cat index - 1)
    const int64_t *tail_off;        // [n_tail+1] rank offsets inside the tail block
    const int64_t *tail_item;       // [n_tail+1] item prefix of the tail category
};

__device__ __forceinline__ uint64_t key_of(const Perm &p, int64_t rs, int64_t rd) {
    return ((uint64_t)p.vertex(rs) << 32) | (uint64_t)p.vertex(rd);
}

__global__ void k_social(SocProg P, uint64_t *keys, int64_t total) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int c = 0;
        while (i >= P.cat_begin[c + 1]) ++c;
        uint32_t cat = (uint32_t)(c + 1);
        int64_t j = i - P.cat_begin[c];
        const uint64_t s = P.seed;
        uint64_t key = 0;
        switch (cat) {
            case S_RING: {  // ring position j -> j+1 in an independent order of the core
                int64_t a = P.ring.vertex(j), b = P.ring.vertex((j + 1) % P.n_core);
                key = key_of(P.perm, a, b);
                break;
            }
            case S_CL:
                key = key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, j, 0))), P.pl_in.sample(u01(rnd(s, cat, j, 1))));
                break;
            case S_SRC0: key = key_of(P.perm, P.b_src + j, P.pl_in.sample(u01(rnd(s, cat, j, 0)))); break;
            case S_SRCX:
                key = key_of(P.perm, P.b_src + P.pl_src.sample(u01(rnd(s, cat, j, 0))),
                             P.pl_in.sample(u01(rnd(s, cat, j, 1))));
                break;
            case S_SNK0: key = key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, j, 0))), P.b_snk + j); break;
            case S_SNKX:
                key = key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, j, 0))),
                             P.b_snk + P.pl_snk.sample(u01(rnd(s, cat, j, 1))));
                break;
            case S_UP: {  // source -> up(k), up(k) -> core
                int64_t k = j >> 1;
                if ((j & 1) == 0)
                    key = key_of(P.perm, P.b_src + (int64_t)(rnd(s, cat, k, 0) % (uint64_t)P.n_src), P.b_up + k);
                else
                    key = key_of(P.perm, P.b_up + k, P.pl_in.sample(u01(rnd(s, cat, k, 1))));
                break;
            }
            case S_DN: {  // core -> dn(k), dn(k) -> sink
                int64_t k = j >> 1;
                if ((j & 1) == 0)
                    key = key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, k, 0))), P.b_dn + k);
                else
                    key = key_of(P.perm, P.b_dn + k, P.b_snk + (int64_t)(rnd(s, cat, k, 1) % (uint64_t)P.n_snk));
                break;
            }
            case S_PAIR: {  // a <-> b, one attachment edge to or from the core
                int64_t k = j / 3, e = j % 3, a = P.b_pair + 2 * k, b = a + 1;
                if (e == 0) key = key_of(P.perm, a, b);
                else if (e == 1) key = key_of(P.perm, b, a);
                else {
                    uint64_t h = rnd(s, cat, k, 2);
                    int64_t m = a + (int64_t)((h >> 1) & 1), cr = P.pl_in.sample(u01(rnd(s, cat, k, 3)));
                    key = (h & 1) ? key_of(P.perm, m, cr) : key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, k, 4))), m);
                }
                break;
            }
            case S_TRI: {  // cycle a->b->c->a or hub a<->b, a<->c; attachment
                int64_t k = j / 5, e = j % 5, a = P.b_tri + 3 * k, b = a + 1, c2 = a + 2;
                bool hub = rnd(s, cat, k, 0) & 1;
                if (e == 4) {
                    uint64_t h = rnd(s, cat, k, 2);
                    int64_t m = a + (int64_t)((h >> 1) % 3);
                    key = (h & 1) ? key_of(P.perm, m, P.pl_in.sample(u01(rnd(s, cat, k, 3))))
                                  : key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, k, 4))), m);
                } else if (hub) {
                    const int64_t sr[4] = {a, b, a, c2}, ds[4] = {b, a, c2, a};
                    key = key_of(P.perm, sr[e], ds[e]);
                } else {
                    const int64_t sr[4] = {a, b, c2, c2}, ds[4] = {b, c2, a, a};
                    key = key_of(P.perm, sr[e], ds[e]);
                }
                break;
            }
            case S_TAIL: {  // ring, chords, one attachment
                int lo = 0, hi = (int)P.n_tail - 1;
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (P.tail_item[mid] <= j) lo = mid; else hi = mid - 1;
                }
                int64_t k = lo, t = j - P.tail_item[k];
                int64_t o = P.b_tail + P.tail_off[k], L = P.tail_off[k + 1] - P.tail_off[k];
                if (t < L) {
                    key = key_of(P.perm, o + t, o + (t + 1) % L);
                } else if (t < L + L / 2) {
                    key = key_of(P.perm, o + (int64_t)(rnd(s, cat, j, 0) % (uint64_t)L),
                                 o + (int64_t)(rnd(s, cat, j, 1) % (uint64_t)L));
                } else {
                    uint64_t h = rnd(s, cat, k, 2);
                    int64_t m = o + (int64_t)((h >> 1) % (uint64_t)L);
                    key = (h & 1) ? key_of(P.perm, m, P.pl_in.sample(u01(rnd(s, cat, k, 3))))
                                  : key_of(P.perm, P.pl_out.sample(u01(rnd(s, cat, k, 4))), m);
                }
                break;
            }
        }
        keys[i] = key;
    }
}

// ---------------------------------------------------------------------------
// keys -> CSR

__global__ void k_flag_unique(const uint64_t *k, int64_t n, uint8_t *flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t x = k[i];
        bool self = (x >> 32) == (x & 0xffffffffull);
        flag[i] = !self && (i == 0 || k[i - 1] != x);
    }
}

// user edge list -> sort keys (src << 32 | dst); ids outside [0, V) are reported
__global__ void k_edge_keys(const int32_t *src, const int32_t *dst, int64_t m, int64_t V, uint64_t *keys,
                            int *bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int32_t s = src[i], d = dst[i];
        const bool ok = s >= 0 && s < V && d >= 0 && d < V;
        if (!ok) atomicOr(bad, 1);
        keys[i] = ok ? ((uint64_t)(uint32_t)s << 32) | (uint32_t)d : 0ull;  // 0 -> 0 is a self-loop, dropped
    }
}

// offsets from keys sorted by src: beg[v] = first index with src >= v
__global__ void k_offsets(const uint64_t *k, int64_t n, int64_t V, int64_t *beg, int32_t *adj) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = i < n ? (int64_t)(k[i] >> 32) : V;
        int64_t p = i > 0 ? (int64_t)(k[i - 1] >> 32) : -1;
        for (int64_t v = p + 1; v <= s && v <= V; ++v) beg[v] = i;
        if (i < n) adj[i] = (int32_t)(k[i] & 0xffffffffull);
    }
}

// offsets of a vertex range [vlo, vlo + vcount) from keys sorted by src:
// beg_out points at beg[vlo], adj_out at the range's first edge, ebase is the
// global index of that edge
__global__ void k_offsets_range(const uint64_t *k, int64_t n, int64_t vlo, int64_t vcount, int64_t *beg_out,
                                int32_t *adj_out, int64_t ebase) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t s = i < n ? (int64_t)(k[i] >> 32) - vlo : vcount;
        int64_t p = i > 0 ? (int64_t)(k[i - 1] >> 32) - vlo : -1;
        for (int64_t v = p + 1; v <= s && v <= vcount; ++v) beg_out[v] = ebase + i;
        if (i < n) adj_out[i] = (int32_t)(k[i] & 0xffffffffull);
    }
}

__global__ void k_swap(const uint64_t *in, uint64_t *out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t x = in[i];
        out[i] = (x << 32) | (x >> 32);
    }
}

static int bits_for(int64_t V) {
    int b = 1;
    while ((1ll << b) < V + 1) ++b;
    return b;
}

// sorts keys (in a, scratch b), drops self-loops/duplicates, builds both CSRs
static int build_csr(uint64_t *a, uint64_t *b, int64_t n, int64_t V, ispan_gen_graph *g) {
    const int vb = bits_for(V);
    const int G = 148 * 8, T = 256;
    size_t tmp_bytes = 0, t2 = 0;
    cub::DoubleBuffer<uint64_t> db(a, b);
    GK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, n, 0, 32 + vb));
    uint8_t *flag = nullptr;
    int64_t *nsel = nullptr;
    GK(cudaMalloc(&flag, std::max<int64_t>(n, 1)));
    GK(cudaMalloc(&nsel, sizeof(int64_t)));
    GK(cub::DeviceSelect::Flagged(nullptr, t2, a, flag, b, nsel, n));
    void *tmp = nullptr;
    GK(cudaMalloc(&tmp, std::max(tmp_bytes, t2) + 256));
    GK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, n, 0, 32 + vb));
    uint64_t *sorted = db.Current(), *other = db.Alternate();
    k_flag_unique<<<G, T>>>(sorted, n, flag);
    GK(cudaGetLastError());
    GK(cub::DeviceSelect::Flagged(tmp, t2, sorted, flag, other, nsel, n));
    int64_t E = 0;
    GK(cudaMemcpy(&E, nsel, sizeof(int64_t), cudaMemcpyDeviceToHost));
    g->V = V;
    g->E = E;
    GK(cudaMalloc(&g->fw_beg, (V + 1) * sizeof(int64_t)));
    GK(cudaMalloc(&g->bw_beg, (V + 1) * sizeof(int64_t)));
    GK(cudaMalloc(&g->fw_adj, std::max<int64_t>(E, 1) * sizeof(int32_t)));
    GK(cudaMalloc(&g->bw_adj, std::max<int64_t>(E, 1) * sizeof(int32_t)));
    k_offsets<<<G, T>>>(other, E, V, g->fw_beg, g->fw_adj);
    GK(cudaGetLastError());
    // transpose: swap halves, sort again (already unique)
    k_swap<<<G, T>>>(other, sorted, E);
    GK(cudaGetLastError());
    cub::DoubleBuffer<uint64_t> db2(sorted, other);
    GK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db2, E, 0, 32 + vb));
    k_offsets<<<G, T>>>(db2.Current(), E, V, g->bw_beg, g->bw_adj);
    GK(cudaGetLastError());
    GK(cudaDeviceSynchronize());
    cudaFree(tmp);
    cudaFree(flag);
    cudaFree(nsel);
    return 0;
}

// Sort a group of keys whose endpoints lie in [vlo, vlo + vcount), drop
// self-loops and duplicates, and write both CSR directions of that vertex
// range into the final arrays at edge bases fw_eb / bw_eb.  Returns the
// group's edge count in *E_out.  a, b: key buffers of n entries.
static int build_csr_range(uint64_t *a, uint64_t *b, int64_t n, int64_t vlo, int64_t vcount, ispan_gen_graph *g,
                           int64_t eb, int64_t *E_out) {
    const int vbits = bits_for(vlo + vcount);
    const int G = 148 * 8, T = 256;
    size_t tmp_bytes = 0, t2 = 0;
    cub::DoubleBuffer<uint64_t> db(a, b);
    GK(cub::DeviceRadixSort::SortKeys(nullptr, tmp_bytes, db, n, 0, 32 + vbits));
    uint8_t *flag = nullptr;
    int64_t *nsel = nullptr;
    GK(cudaMalloc(&flag, std::max<int64_t>(n, 1)));
    GK(cudaMalloc(&nsel, sizeof(int64_t)));
    GK(cub::DeviceSelect::Flagged(nullptr, t2, a, flag, b, nsel, n));
    void *tmp = nullptr;
    GK(cudaMalloc(&tmp, std::max(tmp_bytes, t2) + 256));
    GK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db, n, 0, 32 + vbits));
    uint64_t *sorted = db.Current(), *other = db.Alternate();
    k_flag_unique<<<G, T>>>(sorted, n, flag);
    GK(cudaGetLastError());
    GK(cub::DeviceSelect::Flagged(tmp, t2, sorted, flag, other, nsel, n));
    int64_t E = 0;
    GK(cudaMemcpy(&E, nsel, sizeof(int64_t), cudaMemcpyDeviceToHost));
    k_offsets_range<<<G, T>>>(other, E, vlo, vcount, g->fw_beg + vlo, g->fw_adj + eb, eb);
    GK(cudaGetLastError());
    k_swap<<<G, T>>>(other, sorted, E);
    GK(cudaGetLastError());
    cub::DoubleBuffer<uint64_t> db2(sorted, other);
    GK(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, db2, E, 0, 32 + vbits));
    k_offsets_range<<<G, T>>>(db2.Current(), E, vlo, vcount, g->bw_beg + vlo, g->bw_adj + eb, eb);
    GK(cudaGetLastError());
    GK(cudaDeviceSynchronize());
    cudaFree(tmp);
    cudaFree(flag);
    cudaFree(nsel);
    *E_out = E;
    return 0;
}

static int alloc_keys(int64_t n, uint64_t **a, uint64_t **b) {
    GK(cudaMalloc(a, std::max<int64_t>(n, 1) * sizeof(uint64_t)));
    GK(cudaMalloc(b, std::max<int64_t>(n, 1) * sizeof(uint64_t)));
    return 0;
}

// host-side power-law integer in [lo, hi] with exponent 2 (for cycle lengths)
static int64_t pl_int(std::mt19937_64 &rng, int64_t lo, int64_t hi, double expo) {
    std::uniform_real_distribution<double> U(0.0, 1.0);
    double a = pow((double)lo, 1.0 - expo), b = pow((double)hi + 1.0, 1.0 - expo);
    double x = pow(a + U(rng) * (b - a), 1.0 / (1.0 - expo));
    return std::min<int64_t>(hi, std::max<int64_t>(lo, (int64_t)x));
}

// ---------------------------------------------------------------------------
// R-MAT
__global__ void k_rmat(uint64_t *keys, int64_t m, int scale, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t seed,
                       Perm perm, int permute) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t s = 0, d = 0;
        for (int bit = 0; bit < scale; ++bit) {
            uint32_t r = (uint32_t)(rnd(seed, 77, (uint64_t)i, (uint32_t)bit) >> 32);
            uint64_t sb = r >= tab, db = (r >= ta && r < tab) || r >= tabc;
            s |= sb << bit;
            d |= db << bit;
        }
        if (permute) {
            s = (uint64_t)perm.fwd((int64_t)s);
            d = (uint64_t)perm.fwd((int64_t)d);
        }
        keys[i] = (s << 32) | d;
    }
}

// ---------------------------------------------------------------------------
// web-crawl edge program
enum WebCat : uint32_t { W_RING = 1, W_CORE, W_SRC, W_SNK, W_SCC, W_DAG, W_NCAT };
struct WebProg {
    Perm perm;
    uint64_t seed;
    int64_t n_core, n_src, n_snk, n_scc_v, n_scc;
    int64_t b_src, b_snk, b_scc;
    int64_t core_extra, src_e, snk_e, dag_e;
    int64_t half;  // SCC-block rank where edges to the core stop and edges from it start (an SCC boundary)
    int64_t cat_begin[W_NCAT + 1];
    const int64_t *scc_off;   // [n_scc+1] rank offsets inside the SCC block
    const int64_t *scc_item;  // [n_scc+1] item prefix (ring + chords)
};

__global__ void k_web(WebProg P, uint64_t *keys, int64_t total) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int c = 0;
        while (i >= P.cat_begin[c + 1]) ++c;
        uint32_t cat = (uint32_t)(c + 1);
        int64_t j = i - P.cat_begin[c];
        const uint64_t s = P.seed;
        uint64_t key = 0;
        switch (cat) {
            case W_RING: key = key_of(P.perm, j, (j + 1) % P.n_core); break;
            case W_CORE:
                key = key_of(P.perm, (int64_t)(rnd(s, cat, j, 0) % (uint64_t)P.n_core),
                             (int64_t)(rnd(s, cat, j, 1) % (uint64_t)P.n_core));
                break;
            case W_SRC:  // source -> core or -> planted SCC member
                key = key_of(P.perm, P.b_src + (j % P.n_src),
                             (rnd(s, cat, j, 2) & 3) ? (int64_t)(rnd(s, cat, j, 1) % (uint64_t)P.n_core)
                                                     : P.b_scc + (int64_t)(rnd(s, cat, j, 3) % (uint64_t)P.n_scc_v));
                break;
            case W_SNK:
                key = key_of(P.perm,
                             (rnd(s, cat, j, 2) & 3) ? (int64_t)(rnd(s, cat, j, 1) % (uint64_t)P.n_core)
                                                     : P.b_scc + (int64_t)(rnd(s, cat, j, 3) % (uint64_t)P.n_scc_v),
                             P.b_snk + (j % P.n_snk));
                break;
            case W_SCC: {
                int lo = 0, hi = (int)P.n_scc - 1;
                while (lo < hi) {
                    int mid = (lo + hi + 1) >> 1;
                    if (P.scc_item[mid] <= j) lo = mid; else hi = mid - 1;
                }
                int64_t k = lo, t = j - P.scc_item[k];
                int64_t o = P.b_scc + P.scc_off[k], L = P.scc_off[k + 1] - P.scc_off[k];
                if (t < L) key = key_of(P.perm, o + t, o + (t + 1) % L);
                else
                    key = key_of(P.perm, o + (int64_t)(rnd(s, cat, j, 0) % (uint64_t)L),
                                 o + (int64_t)(rnd(s, cat, j, 1) % (uint64_t)L));
                break;
            }
            case W_DAG: {
                // planted SCCs occupy ranks in topological order; edges go from an
                // earlier SCC vertex to a later one, or between the SCC block and
                // the core in one direction per SCC (earlier half -> core, core ->
                // later half), which keeps every planted SCC separate from the giant
                int64_t x = (int64_t)(rnd(s, cat, j, 0) % (uint64_t)P.n_scc_v);
                int64_t y = (int64_t)(rnd(s, cat, j, 1) % (uint64_t)P.n_scc_v);
                uint64_t h = rnd(s, cat, j, 2);
                if ((h & 7) == 0) {
                    if (x < P.half)
                        key = key_of(P.perm, P.b_scc + x, (int64_t)(rnd(s, cat, j, 3) % (uint64_t)P.n_core));
                    else
                        key = key_of(P.perm, (int64_t)(rnd(s, cat, j, 3) % (uint64_t)P.n_core), P.b_scc + x);
                } else {
                    // map to SCC indices; equal SCC -> chord inside it
                    int lo = 0, hi = (int)P.n_scc - 1;
                    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (P.scc_off[mid] <= x) lo = mid; else hi = mid - 1; }
                    int kx = lo;
                    lo = 0; hi = (int)P.n_scc - 1;
                    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (P.scc_off[mid] <= y) lo = mid; else hi = mid - 1; }
                    int ky = lo;
                    if (kx > ky) { int64_t t = x; x = y; y = t; }
                    key = key_of(P.perm, P.b_scc + x, P.b_scc + y);
                }
                break;
            }
        }
        keys[i] = key;
    }
}

// ---------------------------------------------------------------------------
// batch: graph g has V_g vertices at vbase[g]; R-MAT-like (even g) or planted
// DAG (odd g).  One item per sampled edge; per-graph item prefix.
struct BatchProg {
    uint64_t seed;
    int32_t nseg, max_cycle;
    int32_t g0;             // first graph of this group
    int64_t i0;             // first item of this group
    const int64_t *vbase;   // [nseg+1]
    const int64_t *ibase;   // [nseg+1] item prefix
    const int32_t *scale;   // [nseg] R-MAT scale (2^scale >= V_g)
};

__global__ void k_batch(BatchProg P, uint64_t *keys, int64_t total) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < total; ii += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = ii + P.i0;
        int lo = P.g0, hi = P.nseg - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (P.ibase[mid] <= i) lo = mid; else hi = mid - 1;
        }
        int gidx = lo;
        int64_t j = i - P.ibase[gidx];
        int64_t vb = P.vbase[gidx], V = P.vbase[gidx + 1] - vb;
        uint64_t gs = mix64(P.seed + 0x9e37ull * (uint64_t)gidx);
        uint64_t key;
        if ((gidx & 1) == 0) {
            // R-MAT on 2^scale, folded into [0, V) by modulo, a=.57 b=.19 c=.19
            int sc = P.scale[gidx];
            uint64_t s = 0, d = 0;
            for (int bit = 0; bit < sc; ++bit) {
                uint32_t r = (uint32_t)(rnd(gs, 5, (uint64_t)j, (uint32_t)bit) >> 32);
                uint64_t sb = r >= 3264175145u, db = (r >= 2448131359u && r < 3264175145u) || r >= 4080218931u;
                s |= sb << bit;
                d |= db << bit;
            }
            key = ((uint64_t)(vb + (int64_t)(s % (uint64_t)V)) << 32) | (uint64_t)(vb + (int64_t)(d % (uint64_t)V));
        } else {
            // planted cycles: vertex v's cycle is [start, start+len) where cycles
            // tile [0, V) with lengths from a per-graph hash; items: one ring edge
            // per vertex, then DAG edges from lower to higher cycle
            int64_t cyc_len = 2 + (int64_t)(gs % (uint64_t)(P.max_cycle - 1));
            if (j < V) {
                int64_t start = (j / cyc_len) * cyc_len, len = min(cyc_len, V - start);
                int64_t nxt = start + ((j - start) + 1) % len;
                key = ((uint64_t)(vb + j) << 32) | (uint64_t)(vb + nxt);
            } else {
                int64_t x = (int64_t)(rnd(gs, 6, (uint64_t)j, 0) % (uint64_t)V);
                int64_t y = (int64_t)(rnd(gs, 6, (uint64_t)j, 1) % (uint64_t)V);
                if (x / cyc_len > y / cyc_len) { int64_t t = x; x = y; y = t; }
                key = ((uint64_t)(vb + x) << 32) | (uint64_t)(vb + y);
            }
        }
        keys[ii] = key;
    }
}

}  // namespace

extern "C" {

int ispan_gen_rmat(int device, int scale, int edge_factor, double a, double b, double c, uint64_t seed, int permute,
                   ispan_gen_graph **out) {
    if (!out || scale < 1 || scale > 30 || edge_factor < 1) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -3;
    int64_t V = 1ll << scale, m = (int64_t)edge_factor << scale;
    uint64_t *ka, *kb;
    if (alloc_keys(m, &ka, &kb)) return -2;
    auto th = [](double p) { return (uint32_t)std::min(4294967295.0, std::floor(p * 4294967296.0)); };
    Perm perm = Perm::make(V, seed);
    k_rmat<<<148 * 8, 256>>>(ka, m, scale, th(a), th(a + b), th(a + b + c), seed, perm, permute);
    GK(cudaGetLastError());
    ispan_gen_graph *g = new ispan_gen_graph();
    g->device = device;
    int rc = build_csr(ka, kb, m, V, g);
    cudaFree(ka);
    cudaFree(kb);
    if (rc) { ispan_gen_free(g); return rc; }
    *out = g;
    return 0;
}

int ispan_gen_social(int device, int64_t n, int64_t edges, double giant_frac, double gamma_out, double gamma_in,
                     int64_t n_pair, int64_t n_tri, int64_t n_tail, int32_t max_tail, uint64_t seed,
                     ispan_gen_graph **out) {
    if (!out || n < 16 || n >= (1ll << 31) - 1 || edges < n || max_tail < 4) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -3;
    SocProg P;
    memset(&P, 0, sizeof(P));
    P.seed = seed;
    P.perm = Perm::make(n, seed, (int64_t)(mix64(seed ^ 0x0a11ull) % (uint64_t)std::max<int64_t>(1, (int64_t)(giant_frac * n))));
    std::mt19937_64 rng(seed ^ 0x7a11ull);
    std::vector<int64_t> toff(1, 0), titem(1, 0);
    for (int64_t k = 0; k < n_tail; ++k) {
        int64_t L = pl_int(rng, 4, max_tail, 2.0);
        toff.push_back(toff.back() + L);
        titem.push_back(titem.back() + L + L / 2 + 1);
    }
    P.n_tail = n_tail;
    P.n_tail_v = toff.back();
    P.n_pair = n_pair;
    P.n_tri = n_tri;
    P.n_core = (int64_t)(giant_frac * n);
    P.ring = Perm::make(P.n_core, seed ^ 0x21f6ull);
    int64_t n_triv = n - P.n_core - 2 * n_pair - 3 * n_tri - P.n_tail_v;
    if (P.n_core < 2 || n_triv < 16) return -1;
    P.n_src = n_triv * 45 / 100;
    P.n_snk = n_triv * 45 / 100;
    P.n_up = n_triv * 5 / 100;
    P.n_dn = n_triv - P.n_src - P.n_snk - P.n_up;
    P.b_src = P.n_core;
    P.b_snk = P.b_src + P.n_src;
    P.b_up = P.b_snk + P.n_snk;
    P.b_dn = P.b_up + P.n_up;
    P.b_pair = P.b_dn + P.n_dn;
    P.b_tri = P.b_pair + 2 * n_pair;
    P.b_tail = P.b_tri + 3 * n_tri;
    // edge budget: sources/sinks average 8 edges, the core takes the rest
    int64_t src_x = P.n_src * 7, snk_x = P.n_snk * 7;
    int64_t fixed = P.n_core + P.n_src + src_x + P.n_snk + snk_x + 2 * P.n_up + 2 * P.n_dn + 3 * n_pair + 5 * n_tri +
                    titem.back();
    int64_t cl = std::max<int64_t>(edges - fixed, P.n_core);
    int64_t cnt[S_NCAT] = {0, P.n_core, cl, P.n_src, src_x, P.n_snk, snk_x, 2 * P.n_up, 2 * P.n_dn, 3 * n_pair,
                           5 * n_tri, titem.back()};
    P.cat_begin[0] = 0;
    for (int c = 1; c < S_NCAT; ++c) P.cat_begin[c] = P.cat_begin[c - 1] + cnt[c];
    P.cat_begin[S_NCAT] = INT64_MAX;
    int64_t total = P.cat_begin[S_NCAT - 1];
    // power laws: rank weights (i + i0)^-1/(gamma-1); i0 sets the top degree
    const double b_out = 1.0 / (gamma_out - 1.0), b_in = 1.0 / (gamma_in - 1.0);
    double tot_in = (double)(cl + P.n_src + src_x + P.n_up);
    double tot_out = (double)(cl + P.n_snk + snk_x + P.n_dn);
    // top degrees scale with the edge count like the Twitter crawl that the
    // shape follows: ~770 k out (followees) and ~3 M in (followers) at 1.47 B
    P.pl_out = PowerLaw::fit(P.n_core, b_out, tot_out, 5.2e-4 * (double)edges);
    P.pl_in = PowerLaw::fit(P.n_core, b_in, tot_in, 2.0e-3 * (double)edges);
    P.pl_src = PowerLaw::fit(P.n_src, b_out, (double)src_x, 2000.0);
    P.pl_snk = PowerLaw::fit(P.n_snk, b_in, (double)snk_x, 2000.0);
    int64_t *d_toff = nullptr, *d_titem = nullptr;
    GK(cudaMalloc(&d_toff, toff.size() * 8));
    GK(cudaMalloc(&d_titem, titem.size() * 8));
    GK(cudaMemcpy(d_toff, toff.data(), toff.size() * 8, cudaMemcpyHostToDevice));
    GK(cudaMemcpy(d_titem, titem.data(), titem.size() * 8, cudaMemcpyHostToDevice));
    P.tail_off = d_toff;
    P.tail_item = d_titem;
    uint64_t *ka, *kb;
    if (alloc_keys(total, &ka, &kb)) return -2;
    k_social<<<148 * 16, 256>>>(P, ka, total);
    GK(cudaGetLastError());
    ispan_gen_graph *g = new ispan_gen_graph();
    g->device = device;
    int rc = build_csr(ka, kb, total, n, g);
    cudaFree(ka);
    cudaFree(kb);
    cudaFree(d_toff);
    cudaFree(d_titem);
    if (rc) { ispan_gen_free(g); return rc; }
    {   // core; then pairs, triangles and tail cycles are contiguous from b_pair
        PlantedInfo *pi = new PlantedInfo();
        pi->perm = P.perm;
        pi->n = n;
        pi->n_core = P.n_core;
        pi->block_lo = P.b_pair;
        pi->bnd.push_back(0);
        for (int64_t k = 0; k < n_pair; ++k) pi->bnd.push_back(pi->bnd.back() + 2);
        for (int64_t k = 0; k < n_tri; ++k) pi->bnd.push_back(pi->bnd.back() + 3);
        for (int64_t k = 0; k < n_tail; ++k) pi->bnd.push_back(pi->bnd.back() + (toff[k + 1] - toff[k]));
        g->planted = pi;
    }
    *out = g;
    return 0;
}

int ispan_gen_web(int device, int64_t n, int64_t edges, double giant_frac, double trivial_frac, int32_t min_scc,
                  int32_t max_scc, uint64_t seed, ispan_gen_graph **out) {
    if (!out || n < 64 || n >= (1ll << 31) - 1 || edges < n || min_scc < 2 || max_scc < min_scc) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -3;
    WebProg P;
    memset(&P, 0, sizeof(P));
    P.seed = seed;
    P.n_core = (int64_t)(giant_frac * n);
    P.perm = Perm::make(n, seed, (int64_t)(mix64(seed ^ 0x0a11ull) % (uint64_t)std::max<int64_t>(1, P.n_core)));
    int64_t n_triv = (int64_t)(trivial_frac * n);
    int64_t rest = n - P.n_core - n_triv;
    if (P.n_core < 2 || n_triv < 2 || rest < min_scc) return -1;
    std::mt19937_64 rng(seed ^ 0x3e6ull);
    std::vector<int64_t> off(1, 0), item(1, 0);
    while (off.back() < rest) {
        int64_t L = std::min<int64_t>(pl_int(rng, min_scc, max_scc, 2.0), rest - off.back());
        if (rest - off.back() - L < min_scc && rest - off.back() - L > 0) L = rest - off.back();
        off.push_back(off.back() + L);
        item.push_back(item.back() + L + L / 2);  // ring + chords
    }
    P.n_scc = (int64_t)off.size() - 1;
    P.n_scc_v = rest;
    // no planted SCC may have members on both sides of the split, or it
    // would reach the core and be reached from it (and join the giant)
    P.half = *std::lower_bound(off.begin(), off.end(), rest / 2);
    P.n_src = n_triv / 2;
    P.n_snk = n_triv - P.n_src;
    P.b_src = P.n_core;
    P.b_snk = P.b_src + P.n_src;
    P.b_scc = P.b_snk + P.n_snk;
    P.src_e = P.n_src * 2;
    P.snk_e = P.n_snk * 2;
    P.dag_e = rest * 2;
    int64_t fixed = P.n_core + P.src_e + P.snk_e + item.back() + P.dag_e;
    P.core_extra = std::max<int64_t>(edges - fixed, P.n_core);
    int64_t cnt[W_NCAT] = {0, P.n_core, P.core_extra, P.src_e, P.snk_e, item.back(), P.dag_e};
    P.cat_begin[0] = 0;
    for (int c = 1; c < W_NCAT; ++c) P.cat_begin[c] = P.cat_begin[c - 1] + cnt[c];
    P.cat_begin[W_NCAT] = INT64_MAX;
    int64_t total = P.cat_begin[W_NCAT - 1];
    int64_t *d_off = nullptr, *d_item = nullptr;
    GK(cudaMalloc(&d_off, off.size() * 8));
    GK(cudaMalloc(&d_item, item.size() * 8));
    GK(cudaMemcpy(d_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice));
    GK(cudaMemcpy(d_item, item.data(), item.size() * 8, cudaMemcpyHostToDevice));
    P.scc_off = d_off;
    P.scc_item = d_item;
    uint64_t *ka, *kb;
    if (alloc_keys(total, &ka, &kb)) return -2;
    k_web<<<148 * 16, 256>>>(P, ka, total);
    GK(cudaGetLastError());
    ispan_gen_graph *g = new ispan_gen_graph();
    g->device = device;
    int rc = build_csr(ka, kb, total, n, g);
    cudaFree(ka);
    cudaFree(kb);
    cudaFree(d_off);
    cudaFree(d_item);
    if (rc) { ispan_gen_free(g); return rc; }
    {   // core; the planted SCCs tile the block from b_scc
        PlantedInfo *pi = new PlantedInfo();
        pi->perm = P.perm;
        pi->n = n;
        pi->n_core = P.n_core;
        pi->block_lo = P.b_scc;
        pi->bnd = off;
        g->planted = pi;
    }
    *out = g;
    return 0;
}

int ispan_gen_batch(int device, int32_t nseg, int64_t vmin, int64_t vmax, int32_t ef_min, int32_t ef_max,
                    int32_t max_cycle, uint64_t seed, int64_t *vbase_out, ispan_gen_graph **out) {
    if (!out || !vbase_out || nseg < 1 || vmin < 4 || vmax < vmin || ef_min < 1 || ef_max < ef_min || max_cycle < 2)
        return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -3;
    std::mt19937_64 rng(seed ^ 0xba7cull);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::vector<int64_t> vb(nseg + 1, 0), ib(nseg + 1, 0);
    std::vector<int32_t> sc(nseg, 0);
    for (int g = 0; g < nseg; ++g) {
        int64_t V = (int64_t)std::exp(std::log((double)vmin) + U(rng) * (std::log((double)vmax) - std::log((double)vmin)));
        V = std::max<int64_t>(vmin, std::min<int64_t>(vmax, V));
        vb[g + 1] = vb[g] + V;
        int s = 1;
        while ((1ll << s) < V) ++s;
        sc[g] = s;
        int64_t items;
        if ((g & 1) == 0) items = V * (ef_min + (int64_t)(U(rng) * (ef_max - ef_min + 1)));
        else items = V + V * 2;  // ring edges + DAG edges
        ib[g + 1] = ib[g] + items;
    }
    if (vb[nseg] >= (1ll << 31) - 1) return -1;
    memcpy(vbase_out, vb.data(), (nseg + 1) * sizeof(int64_t));
    const int64_t total = ib[nseg], V = vb[nseg];
    int64_t *d_vb = nullptr, *d_ib = nullptr;
    int32_t *d_sc = nullptr;
    GK(cudaMalloc(&d_vb, vb.size() * 8));
    GK(cudaMalloc(&d_ib, ib.size() * 8));
    GK(cudaMalloc(&d_sc, sc.size() * 4));
    GK(cudaMemcpy(d_vb, vb.data(), vb.size() * 8, cudaMemcpyHostToDevice));
    GK(cudaMemcpy(d_ib, ib.data(), ib.size() * 8, cudaMemcpyHostToDevice));
    GK(cudaMemcpy(d_sc, sc.data(), sc.size() * 4, cudaMemcpyHostToDevice));
    ispan_gen_graph *g = new ispan_gen_graph();
    g->device = device;
    g->V = V;
    // final arrays sized for the sampled edges; the CSR of each group of
    // graphs is built with its keys alone (a group's keys stay under ~1e9),
    // so the whole batch never needs keys for all edges at once
    if (cudaMalloc(&g->fw_beg, (V + 1) * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&g->bw_beg, (V + 1) * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&g->fw_adj, std::max<int64_t>(total, 1) * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&g->bw_adj, std::max<int64_t>(total, 1) * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        ispan_gen_free(g);
        return -2;
    }
    const int64_t kGroupItems = 1000000000ll;
    int64_t gmax = 0;
    for (int g0 = 0; g0 < nseg;) {
        int g1 = g0 + 1;
        while (g1 < nseg && ib[g1 + 1] - ib[g0] <= kGroupItems) ++g1;
        gmax = std::max(gmax, ib[g1] - ib[g0]);
        g0 = g1;
    }
    uint64_t *ka, *kb;
    if (alloc_keys(gmax, &ka, &kb)) { ispan_gen_free(g); return -2; }
    int64_t E = 0;
    int rc = 0;
    for (int g0 = 0; g0 < nseg && !rc;) {
        int g1 = g0 + 1;
        while (g1 < nseg && ib[g1 + 1] - ib[g0] <= kGroupItems) ++g1;
        BatchProg P{seed, nseg, max_cycle, g0, ib[g0], d_vb, d_ib, d_sc};
        int64_t n = ib[g1] - ib[g0];
        k_batch<<<148 * 16, 256>>>(P, ka, n);
        if (cudaGetLastError() != cudaSuccess) { rc = -3; break; }
        int64_t Eg = 0;
        rc = build_csr_range(ka, kb, n, vb[g0], vb[g1] - vb[g0], g, E, &Eg);
        E += Eg;
        g0 = g1;
    }
    g->E = E;
    cudaFree(ka);
    cudaFree(kb);
    cudaFree(d_vb);
    cudaFree(d_ib);
    cudaFree(d_sc);
    if (rc) { ispan_gen_free(g); return rc; }
    *out = g;
    return 0;
}

int ispan_gen_info(const ispan_gen_graph *g, int64_t *V, int64_t *E) {
    if (!g) return -1;
    if (V) *V = g->V;
    if (E) *E = g->E;
    return 0;
}

__global__ void k_narrow(const int64_t *in, int32_t *out, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)in[i];
}

int ispan_gen_copy(const ispan_gen_graph *g, void *fw_beg, int32_t *fw_adj, void *bw_beg, int32_t *bw_adj,
                   int32_t offset_bytes, int32_t to_device) {
    if (!g || (offset_bytes != 4 && offset_bytes != 8)) return -1;
    if (offset_bytes == 4 && g->E >= (1ll << 31)) return -1;
    if (cudaSetDevice(g->device) != cudaSuccess) return -3;
    cudaMemcpyKind k = to_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    int32_t *tmp = nullptr;
    if (offset_bytes == 4) GK(cudaMalloc(&tmp, (g->V + 1) * 4));
    const int64_t *begs[2] = {g->fw_beg, g->bw_beg};
    void *dst[2] = {fw_beg, bw_beg};
    for (int i = 0; i < 2; ++i) {
        if (!dst[i]) continue;
        if (offset_bytes == 8) {
            GK(cudaMemcpy(dst[i], begs[i], (g->V + 1) * 8, k));
        } else {
            k_narrow<<<148 * 4, 256>>>(begs[i], tmp, g->V + 1);
            GK(cudaMemcpy(dst[i], tmp, (g->V + 1) * 4, k));
        }
    }
    if (fw_adj && g->E) GK(cudaMemcpy(fw_adj, g->fw_adj, g->E * 4, k));
    if (bw_adj && g->E) GK(cudaMemcpy(bw_adj, g->bw_adj, g->E * 4, k));
    if (tmp) cudaFree(tmp);
    GK(cudaDeviceSynchronize());
    return 0;
}

int ispan_gen_device_ptrs(const ispan_gen_graph *g, const int64_t **fw_beg, const int32_t **fw_adj,
                          const int64_t **bw_beg, const int32_t **bw_adj) {
    if (!g) return -1;
    if (fw_beg) *fw_beg = g->fw_beg;
    if (fw_adj) *fw_adj = g->fw_adj;
    if (bw_beg) *bw_beg = g->bw_beg;
    if (bw_adj) *bw_adj = g->bw_adj;
    return 0;
}

__global__ void k_extract_beg(const int64_t *beg, int64_t vlo, int64_t n, void *out, int ob) {
    const int64_t b0 = beg[vlo];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t x = beg[vlo + i] - b0;
        if (ob == 8) ((int64_t *)out)[i] = x; else ((int32_t *)out)[i] = (int32_t)x;
    }
}
__global__ void k_extract_adj(const int32_t *adj, int64_t e0, int64_t n, int64_t vlo, int32_t *out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)(adj[e0 + i] - vlo);
}

int ispan_gen_extract(const ispan_gen_graph *g, int64_t vlo, int64_t vhi, void *fw_beg, int32_t *fw_adj,
                      void *bw_beg, int32_t *bw_adj, int32_t offset_bytes, int64_t *E_out) {
    if (!g || vlo < 0 || vhi > g->V || vhi < vlo || (offset_bytes != 4 && offset_bytes != 8)) return -1;
    if (cudaSetDevice(g->device) != cudaSuccess) return -3;
    int64_t f0, f1, b0, b1;
    GK(cudaMemcpy(&f0, g->fw_beg + vlo, 8, cudaMemcpyDeviceToHost));
    GK(cudaMemcpy(&f1, g->fw_beg + vhi, 8, cudaMemcpyDeviceToHost));
    GK(cudaMemcpy(&b0, g->bw_beg + vlo, 8, cudaMemcpyDeviceToHost));
    GK(cudaMemcpy(&b1, g->bw_beg + vhi, 8, cudaMemcpyDeviceToHost));
    if (f1 - f0 != b1 - b0) return -1;  // the range is not closed under edges
    if (E_out) *E_out = f1 - f0;
    const int64_t n = vhi - vlo;
    if (fw_beg) k_extract_beg<<<148, 256>>>(g->fw_beg, vlo, n, fw_beg, offset_bytes);
    if (bw_beg) k_extract_beg<<<148, 256>>>(g->bw_beg, vlo, n, bw_beg, offset_bytes);
    if (fw_adj) k_extract_adj<<<148 * 4, 256>>>(g->fw_adj, f0, f1 - f0, vlo, fw_adj);
    if (bw_adj) k_extract_adj<<<148 * 4, 256>>>(g->bw_adj, b0, b1 - b0, vlo, bw_adj);
    GK(cudaGetLastError());
    GK(cudaDeviceSynchronize());
    return 0;
}

int ispan_gen_from_edges(int device, int64_t V, const int32_t *src, const int32_t *dst, int64_t m,
                         int32_t on_device, ispan_gen_graph **out) {
    if (!out || V < 1 || V >= (1ll << 31) - 1 || m < 0 || (m > 0 && (!src || !dst))) return -1;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return -3;
    const int32_t *ds = src, *dd = dst;
    int32_t *tmp = nullptr;
    if (!on_device && m > 0) {  // stage host edges on the device
        GK(cudaMalloc(&tmp, 2 * m * sizeof(int32_t)));
        GK(cudaMemcpy(tmp, src, m * sizeof(int32_t), cudaMemcpyHostToDevice));
        GK(cudaMemcpy(tmp + m, dst, m * sizeof(int32_t), cudaMemcpyHostToDevice));
        ds = tmp;
        dd = tmp + m;
    }
    uint64_t *ka = nullptr, *kb = nullptr;
    int *bad = nullptr;
    int h_bad = 0;
    if (alloc_keys(m, &ka, &kb)) { cudaFree(tmp); return -2; }
    GK(cudaMalloc(&bad, sizeof(int)));
    GK(cudaMemset(bad, 0, sizeof(int)));
    if (m > 0) {
        k_edge_keys<<<148 * 16, 256>>>(ds, dd, m, V, ka, bad);
        GK(cudaGetLastError());
    }
    GK(cudaMemcpy(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(bad);
    cudaFree(tmp);
    if (h_bad) {  // an id outside [0, V)
        cudaFree(ka);
        cudaFree(kb);
        return -1;
    }
    ispan_gen_graph *g = new ispan_gen_graph();
    g->device = device;
    int rc = build_csr(ka, kb, m, V, g);
    cudaFree(ka);
    cudaFree(kb);
    if (rc) { ispan_gen_free(g); return rc; }
    *out = g;
    return 0;
}

int ispan_gen_planted_labels(const ispan_gen_graph *g, int32_t *labels) {
    if (!g || !labels) return -1;
    if (!g->planted) return -4;
    const PlantedInfo &pi = *g->planted;
    if (cudaSetDevice(g->device) != cudaSuccess) return -3;
    const int64_t nb = (int64_t)pi.bnd.size() - 1;
    int64_t *d_bnd = nullptr;
    int32_t *gmin = nullptr;
    GK(cudaMalloc(&d_bnd, pi.bnd.size() * 8));
    GK(cudaMalloc(&gmin, (nb + 1) * 4));
    GK(cudaMemcpy(d_bnd, pi.bnd.data(), pi.bnd.size() * 8, cudaMemcpyHostToDevice));
    GK(cudaMemset(gmin, 0x7f, (nb + 1) * 4));
    k_planted_min<<<148 * 16, 256>>>(pi.perm, pi.n, pi.n_core, pi.block_lo, d_bnd, nb, gmin);
    GK(cudaGetLastError());
    k_planted_label<<<148 * 16, 256>>>(pi.perm, pi.n, pi.n_core, pi.block_lo, d_bnd, nb, gmin, labels);
    GK(cudaGetLastError());
    GK(cudaDeviceSynchronize());
    cudaFree(d_bnd);
    cudaFree(gmin);
    return 0;
}

int ispan_gen_free(ispan_gen_graph *g) {
    if (!g) return 0;
    delete g->planted;
    cudaSetDevice(g->device);
    cudaFree(g->fw_beg);
    cudaFree(g->bw_beg);
    cudaFree(g->fw_adj);
    cudaFree(g->bw_adj);
    delete g;
    return 0;
}

}  // extern "C"

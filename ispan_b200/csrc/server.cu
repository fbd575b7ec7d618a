// server.cu -- served SCC detection with continuous batching.  Declared in
// include/ispan_b200.h (ispan_server_*).
//
// The reference has no serving mode: it runs one graph per process
// (src/scc_main.cpp:41-47).  Results are those of ispan_scc_run on the graph
// alone: a batch is a disjoint union whose segments never interact (edges
// stay inside their graph, every segment gets its own pivot), and labels are
// translated back to each graph's local ids.
//
// Lanes.  The server runs n_slots lanes, each a context with its own stream
// and worker thread.  A lane whose previous batch is done takes the next
// requests from the head of the queue at once -- while the other lanes'
// batches are still on the device -- so requests that arrive while others
// run are admitted as soon as a lane and memory free up, and their work
// overlaps the running batches on the GPU.  Each lane's persistent stage
// kernels are sized for its share of the SMs (lane.h), which keeps every
// lane's persistent grid co-resident with the others'.
//
// Memory.  The device-memory budget is one allocation made at creation; a
// batch's footprint (every scratch array of its pipeline, the union CSR and
// its tables, exact to the byte for its vertex, edge and graph counts) is
// carved out of it with a first-fit allocator when the batch is admitted and
// handed back when its labels are written.  A request whose footprint alone
// exceeds the budget is refused at submission (ISPAN_ERR_CAPACITY); a batch
// that does not fit the free memory waits for running batches to finish.
// No cudaMalloc or cudaFree runs while batches are in flight (both would
// synchronise the whole device and stall the other lanes).
//
// Requests are taken in arrival order.  A lane takes its share of the queue
// (the queued requests split over the idle lanes), at most max_batch_graphs
// and the per-batch vertex and edge limits, shrunk until it fits the free
// memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ispan_b200.h"
#include "lane.h"

namespace {

int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Req {
    ispan_csr g;
    int32_t *labels = nullptr;
    ispan_request_info info;
};

// First-fit allocator over one device allocation (offsets 256-byte aligned);
// adjacent free ranges are merged on release.
struct Arena {
    size_t cap = 0, used = 0, peak = 0;
    std::map<size_t, size_t> free_;  // offset -> bytes

    void init(size_t bytes) {
        cap = bytes;
        free_.clear();
        free_[0] = bytes;
    }
    bool alloc(size_t bytes, size_t *off) {
        bytes = (bytes + 255) / 256 * 256;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < bytes) continue;
            *off = it->first;
            const size_t rest = it->second - bytes;
            const size_t at = it->first + bytes;
            free_.erase(it);
            if (rest) free_[at] = rest;
            used += bytes;
            peak = std::max(peak, used);
            return true;
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + 255) / 256 * 256;
        used -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

}  // namespace

struct ispan_server {
    ispan_server_config cfg;
    int device = 0;
    std::vector<ispan_ctx *> lanes;
    int64_t capV = 0, capE = 0;     // per-batch limits when a batch holds more than one graph
    int32_t capN = 0;
    size_t cap_bytes = 0;           // per-batch footprint limit (several graphs)
    char *dev_base = nullptr;       // the budget
    Arena arena;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Req> reqs;
    int64_t next_ticket = 1, next_batch = 0;
    int64_t n_batches = 0, n_graphs = 0, n_vertices = 0, n_edges = 0;
    int64_t busy_ns = 0;            // wall time with at least one lane's batch in flight
    int64_t lane_ns = 0;            // sum over batches of their wall time
    int64_t busy_since = 0;
    int active = 0;                 // lanes with a batch in flight
    int idle = 0;                   // lanes waiting for work
    bool stop = false;
    std::vector<std::thread> workers;
    ispan_params params;

    // pack and run one batch on lane c inside its region
    int pack_run(ispan_ctx *c, char *base, size_t bytes, std::vector<ispan_csr> &gs, std::vector<int32_t *> &labs) {
        int64_t V = 0, E = 0, Vh = 0;
        for (const ispan_csr &g : gs) {
            V += g.V;
            E += g.E;
            Vh += g.on_device ? 0 : g.V;
        }
        int rc = lane_bind(c, base, bytes, V, E, (int64_t)gs.size(), Vh);
        if (!rc) rc = ispan_graphs_pack(c, gs.data(), (int32_t)gs.size());
        if (!rc) rc = ispan_graphs_run(c, gs.data(), (int32_t)gs.size(), labs.data(), &params, nullptr);
        lane_unbind(c);
        return rc;
    }

    // the head of the queue this lane takes: its share of the queued
    // requests, within the batch limits, shrunk until it fits free memory;
    // false when nothing can be admitted now
    bool admit(std::vector<int64_t> &take, size_t *off, size_t *bytes) {
        const int64_t share = ((int64_t)pending.size() + idle - 1) / std::max(1, idle);
        int64_t v = 0, e = 0, vh = 0;
        for (int64_t t : pending) {
            if ((int64_t)take.size() >= std::min<int64_t>(capN, std::max<int64_t>(share, 1))) break;
            const Req &r = reqs.at(t);
            const int64_t rh = r.g.on_device ? 0 : r.g.V;
            if (!take.empty() &&
                (v + r.g.V > capV || e + r.g.E > capE ||
                 lane_region_bytes(v + r.g.V, e + r.g.E, (int64_t)take.size() + 1, vh + rh) > cap_bytes))
                break;
            v += r.g.V;
            e += r.g.E;
            vh += rh;
            take.push_back(t);
        }
        while (!take.empty()) {
            *bytes = lane_region_bytes(v, e, (int64_t)take.size(), vh);
            if (arena.alloc(*bytes, off)) return true;
            const Req &r = reqs.at(take.back());
            v -= r.g.V;
            e -= r.g.E;
            vh -= r.g.on_device ? 0 : r.g.V;
            take.pop_back();
        }
        return false;
    }

    void run_batch(ispan_ctx *c, std::vector<int64_t> &take, size_t off, size_t bytes, int64_t t0) {
        std::vector<ispan_csr> gs;
        std::vector<int32_t *> labs;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (int64_t t : take) {
                const Req &r = reqs.at(t);
                gs.push_back(r.g);
                labs.push_back(r.labels);
            }
        }
        std::vector<int> rcs(take.size(), 0);
        int rc = pack_run(c, dev_base + off, bytes, gs, labs);
        if (rc == ISPAN_ERR_ARG && gs.size() > 1) {
            // a malformed graph fails the whole union: run each alone (its
            // footprint is below the batch's) so only that request fails
            for (size_t i = 0; i < gs.size(); ++i) {
                std::vector<ispan_csr> g1(1, gs[i]);
                std::vector<int32_t *> l1(1, labs[i]);
                rcs[i] = pack_run(c, dev_base + off, bytes, g1, l1);
            }
        } else {
            std::fill(rcs.begin(), rcs.end(), rc);
        }
        const int64_t t1 = now_ns();
        std::lock_guard<std::mutex> lk(mu);
        arena.release(off, bytes);
        const int64_t bid = next_batch++;
        ++n_batches;
        lane_ns += t1 - t0;
        if (--active == 0) busy_ns += t1 - busy_since;
        for (size_t i = 0; i < take.size(); ++i) {
            Req &r = reqs.at(take[i]);
            r.info.status = rcs[i] == 0 ? 1 : rcs[i];
            r.info.batch_id = bid;
            r.info.t_done_ns = t1;
            if (rcs[i] == 0) {
                ++n_graphs;
                n_vertices += r.g.V;
                n_edges += r.g.E;
            }
        }
        cv_done.notify_all();
        cv_work.notify_all();  // memory was freed: a waiting lane may admit now
    }

    void loop(int k) {
        ispan_ctx *c = lanes[k];
        for (;;) {
            std::vector<int64_t> take;
            size_t off = 0, bytes = 0;
            int64_t t0 = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                ++idle;
                for (;;) {
                    if (stop && pending.empty()) {
                        --idle;
                        return;
                    }
                    if (!pending.empty()) {
                        if (cfg.max_wait_us > 0 && !stop && (int64_t)pending.size() < capN) {
                            // let a partial batch fill for a bounded time
                            auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(cfg.max_wait_us);
                            cv_work.wait_until(lk, until, [&] { return stop || (int64_t)pending.size() >= capN; });
                            if (pending.empty()) continue;
                        }
                        take.clear();
                        if (admit(take, &off, &bytes)) break;
                    }
                    cv_work.wait(lk);
                }
                --idle;
                for (size_t i = 0; i < take.size(); ++i) pending.pop_front();
                t0 = now_ns();
                if (active++ == 0) busy_since = t0;
                for (int64_t t : take) {
                    Req &r = reqs.at(t);
                    r.info.t_start_ns = t0;
                    r.info.batch_graphs = (int32_t)take.size();
                }
                if (!pending.empty()) cv_work.notify_one();  // the rest is for another lane
            }
            run_batch(c, take, off, bytes, t0);
        }
    }
};

extern "C" {

int ispan_server_create(const ispan_server_config *cfg, ispan_server **out) {
    if (!cfg || !out) return ISPAN_ERR_ARG;
    *out = nullptr;
    const int64_t budget = cfg->hbm_budget_bytes > 0 ? cfg->hbm_budget_bytes : (64ll << 30);
    const int nl = cfg->n_slots > 0 ? cfg->n_slots : 4;
    if (nl > 64) return ISPAN_ERR_ARG;
    ispan_server *s = new ispan_server();
    s->cfg = *cfg;
    s->device = cfg->device;
    s->params = cfg->params;
    // each lane's L2 window would evict the others' maps; lanes run without
    s->params.flags = (s->params.flags | ISPAN_F_NO_L2_WINDOW) & ~(uint32_t)ISPAN_F_LABELS_ON_DEVICE;
    s->capN = cfg->max_batch_graphs > 0 ? cfg->max_batch_graphs : 4096;
    // per-batch size limit: a footprint of half the budget whatever the lane
    // count (a batch's time is set mostly by its slowest graph, so fuller
    // batches serve more requests per unit of time; two such batches still fit
    // side by side), the whole budget with one lane
    const int64_t share = nl == 1 ? budget : budget / 2;
    s->cap_bytes = (size_t)share;
    if (cfg->max_batch_V > 0 && cfg->max_batch_E >= 0) {
        s->capV = cfg->max_batch_V;
        s->capE = cfg->max_batch_E;
        if ((int64_t)lane_region_bytes(s->capV, s->capE, s->capN, s->capV) > budget) {
            delete s;
            return ISPAN_ERR_NOMEM;
        }
    } else {
        s->capV = INT32_MAX - 64;  // the footprint limit decides
        s->capE = INT64_MAX / 4;
        if ((int64_t)lane_region_bytes(1024, 16 * 1024, 1, 1024) > share) {
            delete s;
            return ISPAN_ERR_NOMEM;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        delete s;
        return ISPAN_ERR_NODEV;
    }
    if (cfg->device < 0 || cfg->device >= ndev || cudaSetDevice(cfg->device) != cudaSuccess) {
        delete s;
        return ISPAN_ERR_ARG;
    }
    if (cudaMalloc(&s->dev_base, (size_t)budget) != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return ISPAN_ERR_NOMEM;
    }
    s->arena.init((size_t)budget);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cfg->device);
    // one lane gets every SM; several share 90 % of them, the rest left as
    // slack so the lanes' persistent grids always fit next to each other
    const int sm_share = nl == 1 ? nsm : std::max(1, nsm * 9 / 10 / nl);
    for (int k = 0; k < nl; ++k) {
        ispan_ctx *c = nullptr;
        int rc = ispan_ctx_create(cfg->device, 0, 0, &c);
        if (!rc) rc = lane_set_sm_share(c, sm_share);
        if (!rc) rc = lane_reserve_host(c, s->capN);
        if (rc) {
            if (c) ispan_ctx_destroy(c);
            for (ispan_ctx *d : s->lanes) ispan_ctx_destroy(d);
            cudaFree(s->dev_base);
            delete s;
            return rc;
        }
        s->lanes.push_back(c);
    }
    for (int k = 0; k < nl; ++k) s->workers.emplace_back([s, k] { s->loop(k); });
    *out = s;
    return ISPAN_OK;
}

int ispan_server_limits(const ispan_server *s, int64_t *max_V, int64_t *max_E, int32_t *max_graphs) {
    if (!s) return ISPAN_ERR_ARG;
    if (max_V) *max_V = s->capV;
    if (max_E) *max_E = s->capE;
    if (max_graphs) *max_graphs = s->capN;
    return ISPAN_OK;
}

int ispan_server_submit(ispan_server *s, const ispan_csr *g, int32_t *labels_out, int64_t *ticket) {
    if (!s || !g || !ticket) return ISPAN_ERR_ARG;
    if (g->V < 0 || g->E < 0 || (g->V > 0 && !labels_out)) return ISPAN_ERR_ARG;
    if (g->offset_bytes != 4 && g->offset_bytes != 8) return ISPAN_ERR_ARG;
    if (g->V >= INT32_MAX) return ISPAN_ERR_CAPACITY;
    // a request runs alone if it exceeds the batch limits; it must fit the budget
    if (lane_region_bytes(g->V, g->E, 1, g->on_device ? 0 : g->V) > s->arena.cap) return ISPAN_ERR_CAPACITY;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return ISPAN_ERR_ARG;
    if (s->cfg.max_pending > 0 && (int64_t)s->pending.size() >= s->cfg.max_pending) return ISPAN_ERR_BUSY;
    const int64_t t = s->next_ticket++;
    Req r;
    r.g = *g;
    r.labels = labels_out;
    memset(&r.info, 0, sizeof r.info);
    r.info.t_submit_ns = now_ns();
    s->reqs.emplace(t, r);
    s->pending.push_back(t);
    *ticket = t;
    s->cv_work.notify_one();
    return ISPAN_OK;
}

int ispan_server_poll(ispan_server *s, int64_t ticket, ispan_request_info *info) {
    if (!s) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return ISPAN_ERR_ARG;
    if (info) *info = it->second.info;
    if (it->second.info.status == 0) return 0;
    const int st = it->second.info.status;
    s->reqs.erase(it);  // a finished request is reported once
    return st == 1 ? 1 : st;
}

int ispan_server_wait(ispan_server *s, int64_t ticket, int64_t timeout_us, ispan_request_info *info) {
    if (!s) return ISPAN_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto done = [&] {
        auto it = s->reqs.find(ticket);
        return it == s->reqs.end() || it->second.info.status != 0;
    };
    if (timeout_us < 0) {
        s->cv_done.wait(lk, done);
    } else if (!s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), done)) {
        return 0;
    }
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return ISPAN_ERR_ARG;
    if (info) *info = it->second.info;
    const int st = it->second.info.status;
    s->reqs.erase(it);
    return st == 1 ? 1 : st;
}

int ispan_server_counters(ispan_server *s, int64_t *out, int32_t n) {
    if (!s || !out) return ISPAN_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    // busy time includes the batch in flight now
    const int64_t busy = s->busy_ns + (s->active > 0 ? now_ns() - s->busy_since : 0);
    const int64_t v[10] = {s->n_batches, s->n_graphs, s->n_vertices, s->n_edges, busy,
                           (int64_t)s->pending.size(), s->lane_ns, (int64_t)s->arena.used,
                           (int64_t)s->arena.peak, (int64_t)s->lanes.size()};
    for (int32_t i = 0; i < n && i < 10; ++i) out[i] = v[i];
    return ISPAN_OK;
}

int ispan_server_destroy(ispan_server *s) {
    if (!s) return ISPAN_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    for (std::thread &t : s->workers)  // queued requests are served first
        if (t.joinable()) t.join();
    for (ispan_ctx *c : s->lanes) ispan_ctx_destroy(c);
    if (s->dev_base) {
        cudaSetDevice(s->device);
        cudaFree(s->dev_base);
    }
    delete s;
    return ISPAN_OK;
}

}  // extern "C"

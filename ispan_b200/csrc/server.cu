// server.cu -- served SCC detection: requests (one graph each) are queued,
// gathered into batches while the device works on the previous batch
// (continuous batching), and run as one disjoint union per batch through
// the two phases of ispan_scc_run_graphs (ispan_graphs_pack, then
// ispan_graphs_run).  Declared in include/ispan_b200.h (ispan_server_*).
//
// The reference has no serving mode: it runs one graph per process
// (src/scc_main.cpp:41-47).  Results are those of ispan_scc_run on the graph
// alone: the union's segments never interact (edges stay inside their
// graph, every segment gets its own pivot), and labels are translated back to
// each graph's local ids.
//
// Admission: the budget is split between the batch slots, each a context
// plus its union buffers; a request larger than one batch is refused at
// submission (ISPAN_ERR_CAPACITY), and the queue may be bounded
// (ISPAN_ERR_BUSY).  Requests run in arrival order; a batch takes requests
// from the head of the queue while they fit.  While one slot's batch runs,
// another slot packs the next batch (host copies and the pack kernels on its
// own stream), so arrivals join the device work as soon as a slot frees.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/ispan_b200.h"

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

// device bytes of a server whose batches hold up to V vertices, E edges and
// n graphs: the context plus the union CSR and its staging tables
int64_t server_bytes(int64_t V, int64_t E, int64_t n) {
    return ispan_ctx_bytes(V, E) + 2 * 8 * (V + 1) + 2 * 4 * E + 2 * 8 * (V + n) + 4 * 8 * (n + 1) + 96 * n;
}

}  // namespace

struct ispan_server {
    ispan_server_config cfg;
    std::vector<ispan_ctx *> ctx;   // one per batch slot
    int64_t capV = 0, capE = 0;     // per batch (one slot)
    int32_t capN = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<int64_t> pending;
    std::unordered_map<int64_t, Req> reqs;
    int64_t next_ticket = 1, next_batch = 0;
    int64_t n_batches = 0, n_graphs = 0, n_vertices = 0, n_edges = 0, busy_ns = 0;
    bool stop = false;
    bool device_busy = false;       // a slot's pipeline is on the device
    std::mutex dev_mu;              // one pipeline on the device at a time
    std::vector<std::thread> workers;

    bool batch_full() const {
        int64_t v = 0, e = 0, k = 0;
        for (int64_t t : pending) {
            const Req &r = reqs.at(t);
            if (k + 1 > capN || v + r.g.V > capV || e + r.g.E > capE) return true;
            v += r.g.V;
            e += r.g.E;
            ++k;
        }
        return false;
    }

    // pack on this slot's context (overlapping another slot's run), then run
    // when the device is free
    int pack_run(ispan_ctx *c, std::vector<ispan_csr> &gs, std::vector<int32_t *> &labs) {
        int rc = ispan_graphs_pack(c, gs.data(), (int32_t)gs.size());
        if (rc) return rc;
        std::lock_guard<std::mutex> dev(dev_mu);
        {
            std::lock_guard<std::mutex> lk(mu);
            device_busy = true;
        }
        rc = ispan_graphs_run(c, gs.data(), (int32_t)gs.size(), labs.data(), &cfg.params, nullptr);
        {
            std::lock_guard<std::mutex> lk(mu);
            device_busy = false;
        }
        cv_work.notify_all();  // an idle device lets a waiting slot take a batch
        return rc;
    }

    void run_batch(ispan_ctx *c, std::vector<int64_t> &take) {
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
        const int64_t t0 = now_ns();
        std::vector<int> rcs(take.size(), 0);
        int rc = pack_run(c, gs, labs);
        if (rc == ISPAN_ERR_ARG && gs.size() > 1) {
            // a malformed graph fails the whole union: run each alone so only
            // that request reports the error
            for (size_t i = 0; i < gs.size(); ++i) {
                std::vector<ispan_csr> g1(1, gs[i]);
                std::vector<int32_t *> l1(1, labs[i]);
                rcs[i] = pack_run(c, g1, l1);
            }
        } else {
            std::fill(rcs.begin(), rcs.end(), rc);
        }
        const int64_t t1 = now_ns();
        std::lock_guard<std::mutex> lk(mu);
        const int64_t bid = next_batch++;
        ++n_batches;
        busy_ns += t1 - t0;
        for (size_t i = 0; i < take.size(); ++i) {
            Req &r = reqs.at(take[i]);
            r.info.status = rcs[i] == 0 ? 1 : rcs[i];
            r.info.batch_id = bid;
            r.info.batch_graphs = (int32_t)take.size();
            r.info.t_start_ns = t0;
            r.info.t_done_ns = t1;
            if (rcs[i] == 0) {
                ++n_graphs;
                n_vertices += r.g.V;
                n_edges += r.g.E;
            }
        }
        cv_done.notify_all();
    }

    // A slot takes a batch when the device is idle (latency) or a full batch
    // is queued (throughput: it packs while the running batch computes).
    void loop(int slot) {
        ispan_ctx *c = ctx[slot];
        for (;;) {
            std::vector<int64_t> take;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || (!pending.empty() && (!device_busy || batch_full())); });
                if (stop && pending.empty()) return;
                if (cfg.max_wait_us > 0 && !stop) {
                    // let a partial batch fill for a bounded time
                    auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(cfg.max_wait_us);
                    cv_work.wait_until(lk, until, [&] { return stop || batch_full(); });
                }
                int64_t v = 0, e = 0;
                while (!pending.empty() && (int32_t)take.size() < capN) {
                    const Req &r = reqs.at(pending.front());
                    if (!take.empty() && (v + r.g.V > capV || e + r.g.E > capE)) break;
                    v += r.g.V;
                    e += r.g.E;
                    take.push_back(pending.front());
                    pending.pop_front();
                }
            }
            if (!take.empty()) run_batch(c, take);
        }
    }
};

extern "C" {

int ispan_server_create(const ispan_server_config *cfg, ispan_server **out) {
    if (!cfg || !out) return ISPAN_ERR_ARG;
    *out = nullptr;
    ispan_server *s = new ispan_server();
    s->cfg = *cfg;
    const int64_t budget = cfg->hbm_budget_bytes > 0 ? cfg->hbm_budget_bytes : (64ll << 30);
    const int nslots = cfg->n_slots > 0 ? cfg->n_slots : 2;
    const int64_t share = budget / nslots;
    s->capN = cfg->max_batch_graphs > 0 ? cfg->max_batch_graphs : 4096;
    if (cfg->max_batch_V > 0 && cfg->max_batch_E >= 0) {
        s->capV = cfg->max_batch_V;
        s->capE = cfg->max_batch_E;
        if (server_bytes(s->capV, s->capE, s->capN) > share) {
            delete s;
            return ISPAN_ERR_NOMEM;
        }
    } else {
        // the largest batch at 16 edges per vertex that fits a slot's share
        int64_t lo = 0, hi = (int64_t)INT32_MAX - 64;
        while (lo < hi) {
            int64_t mid = (lo + hi + 1) / 2;
            if (server_bytes(mid, 16 * mid, s->capN) <= share) lo = mid; else hi = mid - 1;
        }
        if (lo < 1024) {
            delete s;
            return ISPAN_ERR_NOMEM;
        }
        s->capV = lo;
        s->capE = 16 * lo;
    }
    for (int k = 0; k < nslots; ++k) {
        ispan_ctx *c = nullptr;
        int rc = ispan_ctx_create(cfg->device, s->capV, s->capE, &c);
        if (rc) {
            for (ispan_ctx *d : s->ctx) ispan_ctx_destroy(d);
            delete s;
            return rc;
        }
        s->ctx.push_back(c);
    }
    for (int k = 0; k < nslots; ++k) s->workers.emplace_back([s, k] { s->loop(k); });
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
    if (g->V > s->capV || g->E > s->capE) return ISPAN_ERR_CAPACITY;
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
    const int64_t v[6] = {s->n_batches, s->n_graphs, s->n_vertices, s->n_edges, s->busy_ns,
                          (int64_t)s->pending.size()};
    for (int32_t i = 0; i < n && i < 6; ++i) out[i] = v[i];
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
    for (ispan_ctx *c : s->ctx) ispan_ctx_destroy(c);
    delete s;
    return ISPAN_OK;
}

}  // extern "C"

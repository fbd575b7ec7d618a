// ref_capi.cpp -- TEST INFRASTRUCTURE.  In-process C entry point over the
// reference's unmodified scc_detection (src/scc_core.cpp:27, declared at
// src/scc_common.h:15-23), so the reference's own OpenMP pipeline can be
// timed on host arrays without writing CSR files.  The reference's graph
// class (src/graph.h:9-31) has public raw pointers and a default constructor,
// so the caller's int32 arrays are attached to it directly.  The link-time
// hook get_scc_result (src/load_print.cpp:24) copies the [V+1] scc_id codes
// out to the caller.  Built only into oracle/_ref/libispan_ref.so.
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <fcntl.h>
#include <unistd.h>
#include "graph.h"
#include "scc_common.h"

static thread_local index_t *g_scc_dst = nullptr;

void get_scc_result(index_t *scc_id, index_t vert_count)
{
    if (g_scc_dst) memcpy(g_scc_dst, scc_id, ((size_t)vert_count + 1) * sizeof(index_t));
}

void print_time_result(index_t, double *) {}

graph *graph_load(const char *a, const char *b, const char *c, const char *d, double *avg_time)
{
    for (int i = 0; i < 15; ++i) avg_time[i] = 0.0;
    return new graph(a, b, c, d);
}

#ifndef ISPAN_REF64
extern "C" int ispan_ref_run(int32_t V, int32_t E, int32_t *fw_beg, int32_t *fw_adj,
                             int32_t *bw_beg, int32_t *bw_adj, int threads, int alpha,
                             int beta, int gamma, double theta, double *avg_time15,
                             int32_t *scc_id_out, int quiet)
#else
// The wide build (oracle/Makefile ref64): the reference compiled with its
// integer types (src/util.h:17-21) widened to 64 bits, for graphs whose edge
// count needs 64-bit offsets.
extern "C" int ispan_ref_run64(int64_t V, int64_t E, int64_t *fw_beg, int64_t *fw_adj,
                               int64_t *bw_beg, int64_t *bw_adj, int threads, int alpha,
                               int beta, int gamma, double theta, double *avg_time15,
                               int64_t *scc_id_out, int quiet)
#endif
{
    static_assert(sizeof(*fw_beg) == sizeof(index_t), "offset width of the compiled reference");
    static_assert(sizeof(*fw_adj) == sizeof(vertex_t), "vertex id width of the compiled reference");
    graph g;
    g.fw_beg_pos = (index_t *)fw_beg;
    g.fw_csr = (vertex_t *)fw_adj;
    g.bw_beg_pos = (index_t *)bw_beg;
    g.bw_csr = (vertex_t *)bw_adj;
    g.weight = nullptr;
    g.vert_count = V;
    g.edge_count = E;
    g.src_list = nullptr;
    g.src_count = 0;
    int saved = -1;
    if (quiet) { // the pipeline prints stage times to stdout (OUTPUT_TIME, util.h:29)
        fflush(stdout);
        saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        if (dn >= 0) { dup2(dn, 1); close(dn); }
    }
    g_scc_dst = (index_t *)scc_id_out;
    scc_detection(&g, alpha, beta, gamma, theta, threads, avg_time15);
    g_scc_dst = nullptr;
    fflush(stdout);
    if (saved >= 0) { dup2(saved, 1); close(saved); }
    return 0;
}

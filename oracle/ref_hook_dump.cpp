// ref_hook_dump.cpp -- TEST INFRASTRUCTURE.  Link-time replacement for the
// reference's src/load_print.cpp (graph_load at :6-22, get_scc_result at
// :24-60, print_time_result at :62-92) used to build oracle/_ref/ispan_dump:
// the same CLI (src/scc_main.cpp) and pipeline (src/scc_core.cpp), compiled
// unmodified from the reference tree, but the per-vertex scc_id array that
// the pipeline hands to get_scc_result (scc_core.cpp:1076) is written to the
// file named by $ISPAN_DUMP ([V+1] int32, the reference's own codes).
#include <cstdio>
#include <cstdlib>
#include "graph.h"
#include "util.h"

graph *graph_load(const char *fw_beg_file, const char *fw_csr_file,
                  const char *bw_beg_file, const char *bw_csr_file, double *avg_time)
{
    graph *g = new graph(fw_beg_file, fw_csr_file, bw_beg_file, bw_csr_file);
    for (int i = 0; i < 15; ++i) avg_time[i] = 0.0;
    return g;
}

void get_scc_result(index_t *scc_id, index_t vert_count)
{
    const char *path = getenv("ISPAN_DUMP");
    if (!path) return;
    FILE *f = fopen(path, "wb");
    if (!f) { perror(path); return; }
    size_t n = (size_t)vert_count + 1;
    if (fwrite(scc_id, sizeof(index_t), n, f) != n) perror(path);
    fclose(f);
}

void print_time_result(index_t run_times, double *avg_time)
{
    // machine-readable mean stage times in ms, slot meanings of
    // src/scc_core.cpp:1037-1053 (0 trim, 1 elephant, 2 mice, 3 total, ...)
    printf("ISPAN_TIMES_MS");
    for (int i = 0; i < 15; ++i)
        printf(" %.6f", run_times > 0 ? avg_time[i] / run_times * 1000.0 : 0.0);
    printf("\n");
}

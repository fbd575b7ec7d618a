/*
 * ispan_oracle.c -- CPU oracle for the iSpan SCC pipeline (TEST INFRASTRUCTURE).
 *
 * Serial restatement of src/scc_core.cpp:27-1094 of iSpan with thread_count=1,
 * so every "per-thread slice" of the reference is the whole range.  The stage
 * order, stop rules and data structures follow the reference; only the quirks
 * that make the reference's answer wrong or ambiguous are fixed (marked FIX).
 * Plus an independent iterative Tarjan used to pin everything to the exact
 * SCC partition.  Never linked into the product.
 */
#include "ispan_oracle.h"
#include <stdlib.h>
#include <string.h>

#define ACT 0 /* scc_id == 0: unassigned, as in the reference */

static inline int64_t outdeg(const oc_graph *g, int64_t v) { return g->fw_beg[v + 1] - g->fw_beg[v]; }
static inline int64_t indeg(const oc_graph *g, int64_t v) { return g->bw_beg[v + 1] - g->bw_beg[v]; }

/* ---------------------------------------------------------------------------
 * Working state of one run (src/scc_core.cpp:56-125).
 * sid    : scc_id of the reference (0 active, 1 giant, -1..-4 trim classes,
 *          otherwise mice).  Held as int64 so a mice label can be pivot+2.
 * group  : FIX(Q2): component key per vertex, kept apart from the class code.
 */
typedef struct {
    const oc_graph *g;
    int64_t *sid;
    int64_t *group;
    int32_t *fw_sa, *bw_sa;
    int64_t *color;
    int64_t *Q, *tmpq, *ring;
    int64_t fq;
    int quirks;
    int nonterminating; /* set when the reproduced reference would loop forever */
} st_t;

/* trim_1_first (src/trim_1_gfq.h:9-33): zero full out- or in-degree. */
static void trim_1_first(st_t *s, oc_stats *st)
{
    const oc_graph *g = s->g;
    for (int64_t v = 0; v < g->V; ++v)
        if (outdeg(g, v) == 0 || indeg(g, v) == 0) {
            s->sid[v] = -1;
            s->group[v] = v;
            st->n_trim1++;
        }
}

/* generate_frontier_queue (src/trim_1_gfq.h:486-529): ordered compaction. */
static void generate_frontier_queue(st_t *s)
{
    s->fq = 0;
    for (int64_t v = 0; v < s->g->V; ++v)
        if (s->sid[v] == ACT) s->Q[s->fq++] = v;
}

/* pivot_selection_from_fq (src/scc_common.h:92-150): first argmax of
 * outdeg*indeg over the worklist.  FIX(Q4): 64-bit product. */
static int64_t pivot_selection_from_fq(st_t *s)
{
    int64_t best = 0, piv = -1;
    for (int64_t i = 0; i < s->fq; ++i) {
        int64_t v = s->Q[i];
        int64_t m = outdeg(s->g, v) * indeg(s->g, v);
        if (s->quirks & OC_Q4) /* the reference's wrapping int32 product */
            m = (int32_t)((uint32_t)outdeg(s->g, v) * (uint32_t)indeg(s->g, v));
        if (m > best) { best = m; piv = v; }
    }
    if (s->quirks & OC_Q8) return piv < 0 ? 0 : piv;
    /* FIX(Q8): the reference defaults the pivot to vertex 0 even when 0 is
     * already trimmed; here an empty or all-zero-product worklist yields the
     * first worklist vertex, or no pivot when the worklist is empty. */
    if (piv < 0 && s->fq > 0) piv = s->Q[0];
    return piv;
}

/* fw_bfs_fq_queue (src/fw_bw.h:396-698), serial: synchronous top-down over the
 * current queue, "Rsync" bottom-up over the worklist that stops at the first
 * visited in-neighbour of any level, and the asynchronous top-down ring queue
 * that runs to exhaustion.  Switch rules at fw_bw.h:576-624. */
static int32_t fw_bfs_fq_queue(st_t *s, int64_t root, int alpha, int beta, int gamma, double avg_degree)
{
    const oc_graph *g = s->g;
    int32_t level = 0;
    int64_t *tq = s->tmpq, qsize = 1, visited = 0;
    int64_t *nq = s->ring; /* next-level queue (thread_queue) */
    int is_td = 1, is_tdq = 0;
    s->fw_sa[root] = 0;
    tq[0] = root;
    for (;;) {
        int64_t frontier = 0;
        if (is_td) {
            for (int64_t i = 0; i < qsize; ++i) {
                int64_t v = tq[i];
                if (s->sid[v] == ACT && s->fw_sa[v] != -1)
                    for (int64_t e = g->fw_beg[v]; e < g->fw_beg[v + 1]; ++e) {
                        int64_t w = g->fw_adj[e];
                        if (s->sid[w] == ACT && s->fw_sa[w] == -1) {
                            s->fw_sa[w] = level + 1;
                            nq[frontier++] = w;
                        }
                    }
            }
        } else if (!is_tdq) {
            for (int64_t i = 0; i < s->fq; ++i) {
                int64_t v = s->Q[i];
                if (s->sid[v] == ACT && s->fw_sa[v] == -1)
                    for (int64_t e = g->bw_beg[v]; e < g->bw_beg[v + 1]; ++e) {
                        int64_t u = g->bw_adj[e];
                        if (s->sid[u] == ACT && s->fw_sa[u] != -1) {
                            s->fw_sa[v] = level + 1;
                            frontier++;
                            break;
                        }
                    }
            }
        } else {
            /* ring queue of the async top-down mode (fw_bw.h:506-544); it
             * never counts a frontier, so the level loop ends after it. */
            int64_t head = 0, tail = 0, cap = g->V + 1;
            for (int64_t i = 0; i < qsize; ++i) nq[tail++] = tq[i];
            while (head != tail) {
                int64_t v = nq[head++];
                if (head == cap) head = 0;
                for (int64_t e = g->fw_beg[v]; e < g->fw_beg[v + 1]; ++e) {
                    int64_t w = g->fw_adj[e];
                    if (s->sid[w] == ACT && s->fw_sa[w] == -1) {
                        nq[tail++] = w;
                        if (tail == cap) tail = 0;
                        s->fw_sa[w] = level + 1;
                    }
                }
            }
        }
        visited += frontier;
        if (frontier == 0) break;
        if (is_td) {
            double ef = (double)frontier * avg_degree;
            double er = (double)(s->fq - visited) * avg_degree;
            if (!is_tdq && er / alpha < ef) is_td = 0;
        } else if ((!is_tdq && (s->fq * 1.0 / beta) > frontier) || (!is_tdq && level > gamma)) {
            frontier = 0;
            for (int64_t i = 0; i < s->fq; ++i) {
                int64_t v = s->Q[i];
                if (s->sid[v] == ACT && s->fw_sa[v] == level + 1) nq[frontier++] = v;
            }
            is_tdq = 1;
        }
        if (is_td || is_tdq) { /* get_queue (trim_1_gfq.h:460-483) */
            memcpy(tq, nq, (size_t)frontier * sizeof(int64_t));
            qsize = frontier;
        }
        level++;
    }
    return level;
}

/* bw_gfq_from_fw (src/trim_1_gfq.h:583-633): worklist of fw_sa != -1. */
static int64_t bw_gfq_from_fw(st_t *s, int64_t *out)
{
    int64_t n = 0;
    for (int64_t i = 0; i < s->fq; ++i)
        if (s->fw_sa[s->Q[i]] != -1) out[n++] = s->Q[i];
    return n;
}

/* bw_bfs_fq_queue (src/fw_bw.h:944-1248): reachability to the pivot inside
 * the forward set; members get scc_id = 1. */
static int32_t bw_bfs_fq_queue(st_t *s, int64_t root, const int64_t *FQ, int64_t ffq,
                               int alpha, int beta, int gamma, double avg_degree, int64_t *tq)
{
    const oc_graph *g = s->g;
    int32_t level = 0;
    int64_t qsize = 1, visited = 0;
    int64_t *nq = s->ring;
    int is_td = 1, is_tdq = 0;
    s->bw_sa[root] = 0;
    s->sid[root] = 1; /* fw_bw.h:974, unconditionally (only Q8 can pass an inactive root) */
    tq[0] = root;
    for (;;) {
        int64_t frontier = 0;
        if (is_td) {
            for (int64_t i = 0; i < qsize; ++i) {
                int64_t v = tq[i];
                if (s->sid[v] == 1)
                    for (int64_t e = g->bw_beg[v]; e < g->bw_beg[v + 1]; ++e) {
                        int64_t u = g->bw_adj[e];
                        if (s->sid[u] == ACT && s->bw_sa[u] == -1 && s->fw_sa[u] != -1) {
                            s->bw_sa[u] = level + 1;
                            nq[frontier++] = u;
                            s->sid[u] = 1;
                        }
                    }
            }
        } else if (!is_tdq) {
            for (int64_t i = 0; i < ffq; ++i) {
                int64_t v = FQ[i];
                if (s->sid[v] == ACT && s->fw_sa[v] != -1)
                    for (int64_t e = g->fw_beg[v]; e < g->fw_beg[v + 1]; ++e) {
                        int64_t w = g->fw_adj[e];
                        if (s->sid[w] == 1) {
                            s->bw_sa[v] = level + 1;
                            frontier++;
                            s->sid[v] = 1;
                            break;
                        }
                    }
            }
        } else {
            int64_t head = 0, tail = 0, cap = g->V + 1;
            for (int64_t i = 0; i < qsize; ++i) nq[tail++] = tq[i];
            while (head != tail) {
                int64_t v = nq[head++];
                if (head == cap) head = 0;
                for (int64_t e = g->bw_beg[v]; e < g->bw_beg[v + 1]; ++e) {
                    int64_t u = g->bw_adj[e];
                    if (s->sid[u] == ACT && s->bw_sa[u] == -1 && s->fw_sa[u] != -1) {
                        nq[tail++] = u;
                        if (tail == cap) tail = 0;
                        s->sid[u] = 1;
                        s->bw_sa[u] = level + 1;
                    }
                }
            }
        }
        visited += frontier;
        if (frontier == 0) break;
        if (is_td) {
            double ef = (double)frontier * avg_degree;
            double er = (double)(ffq - visited) * avg_degree;
            if (!is_tdq && er / alpha < ef) is_td = 0;
        } else if ((!is_tdq && (ffq * 1.0 / beta) > frontier) || (!is_tdq && level > gamma)) {
            frontier = 0;
            for (int64_t i = 0; i < ffq; ++i) {
                int64_t v = FQ[i];
                if (s->sid[v] == 1 && s->bw_sa[v] == level + 1) nq[frontier++] = v;
            }
            is_tdq = 1;
        }
        if (is_td || is_tdq) {
            memcpy(tq, nq, (size_t)frontier * sizeof(int64_t));
            qsize = frontier;
        }
        level++;
    }
    return level;
}

/* scan helper shared by the trims: first active neighbour other than skip_a /
 * skip_b; returns count of distinct active neighbours seen, capped at cap. */

/* trim_1_from_fq_gfq (src/trim_1_gfq.h:365-458): peel worklist vertices with
 * no active out- or in-neighbour other than themselves, then compact the
 * worklist to the still-active vertices. */
static void trim_1_from_fq_gfq(st_t *s, oc_stats *st)
{
    const oc_graph *g = s->g;
    int64_t n = 0;
    for (int64_t i = 0; i < s->fq; ++i) {
        int64_t v = s->Q[i];
        if (s->sid[v] != ACT) continue;
        int has = 0;
        for (int64_t e = g->fw_beg[v]; e < g->fw_beg[v + 1]; ++e) {
            int64_t w = g->fw_adj[e];
            if (s->sid[w] == ACT && w != v) { has = 1; break; }
        }
        if (has) {
            has = 0;
            for (int64_t e = g->bw_beg[v]; e < g->bw_beg[v + 1]; ++e) {
                int64_t w = g->bw_adj[e];
                if (s->sid[w] == ACT && w != v) { has = 1; break; }
            }
        }
        if (!has) {
            s->sid[v] = -1;
            s->group[v] = v;
            st->n_trim1++;
        }
    }
    for (int64_t i = 0; i < s->fq; ++i)
        if (s->sid[s->Q[i]] == ACT) s->Q[n++] = s->Q[i];
    s->fq = n;
    st->trim1_passes++;
}

/* distinct active neighbours of v in one direction, excluding x1 and x2,
 * stopping at cap; the first two are returned in n1/n2. */
static int nbrs(const st_t *s, int fw, int64_t v, int64_t x1, int64_t x2, int cap, int64_t *n1, int64_t *n2)
{
    const oc_graph *g = s->g;
    const int64_t *beg = fw ? g->fw_beg : g->bw_beg;
    const int32_t *adj = fw ? g->fw_adj : g->bw_adj;
    int d = 0;
    for (int64_t e = beg[v]; e < beg[v + 1]; ++e) {
        int64_t w = adj[e];
        if (s->sid[w] != ACT || w == x1 || w == x2) continue;
        if (d == 0) { *n1 = w; d = 1; }
        else if (d == 1 && w != *n1) { *n2 = w; d = 2; }
        else if (d == 2 && w != *n1 && w != *n2) { d = 3; }
        if (d >= cap) break;
    }
    return d;
}

static int64_t min3(int64_t a, int64_t b, int64_t c) { int64_t m = a < b ? a : b; return m < c ? m : c; }

/* trim_2_from_fq (src/trim_2_3.h:146-283): a vertex with a single distinct
 * active out-neighbour whose single distinct active out-neighbour is the
 * vertex itself forms a sink 2-cycle; the same for in-neighbours.
 * FIX(Q9): the scc_id guard that the reference comments out is applied (the
 * outcome is identical; the guard only skips dead work). */
static void trim_2_from_fq(st_t *s, oc_stats *st)
{
    for (int64_t i = 0; i < s->fq; ++i) {
        int64_t v = s->Q[i], a = -1, b = -1, c = -1, d = -1;
        if (s->sid[v] != ACT) continue;
        for (int dir = 1; dir >= 0; --dir) {
            if (nbrs(s, dir, v, v, v, 2, &a, &b) == 1 &&
                nbrs(s, dir, a, a, a, 2, &c, &d) == 1 && c == v) {
                s->sid[v] = s->sid[a] = -2;
                s->group[v] = s->group[a] = v < a ? v : a;
                st->n_trim2 += 2;
                break;
            }
        }
    }
}

/* trim_3_1_from_fq (src/trim_2_3.h:482-677): A->B->C->A with A, B, C each
 * having a single distinct active successor outside {self, previous}, in both
 * edge directions. */
static void trim_3_1_from_fq(st_t *s, oc_stats *st)
{
    for (int64_t i = 0; i < s->fq; ++i) {
        int64_t v = s->Q[i];
        if (s->sid[v] != ACT) continue;
        for (int dir = 1; dir >= 0; --dir) {
            int64_t B = -1, x = -1, C = -1, A2 = -1;
            if (nbrs(s, dir, v, v, v, 2, &B, &x) != 1 || B == v) continue;
            if (nbrs(s, dir, B, B, v, 2, &C, &x) != 1) continue;
            if (nbrs(s, dir, C, C, B, 2, &A2, &x) == 1 && A2 == v) {
                s->sid[v] = s->sid[B] = s->sid[C] = -3;
                s->group[v] = s->group[B] = s->group[C] = min3(v, B, C);
                st->n_trim3_cycle += 3;
                break;
            }
        }
    }
}

/* trim_3_2_from_fq (src/trim_2_3.h:881-1080): hub A with exactly two distinct
 * active successors B, C, each of which has A as its only active successor
 * outside {B, C}; in both edge directions. */
static void trim_3_2_from_fq(st_t *s, oc_stats *st)
{
    for (int64_t i = 0; i < s->fq; ++i) {
        int64_t v = s->Q[i];
        if (s->sid[v] != ACT) continue;
        for (int dir = 1; dir >= 0; --dir) {
            int64_t B = -1, C = -1, a = -1, x = -1;
            if (nbrs(s, dir, v, v, v, 3, &B, &C) != 2) continue;
            /* the reference stops at the second qualifying edge here even if
             * it repeats the first (trim_2_3.h:948-957); with distinct
             * neighbours, as counted by nbrs, the outcome is the same */
            if (nbrs(s, dir, B, B, C, 2, &a, &x) != 1 || a != v) continue;
            if (nbrs(s, dir, C, C, B, 2, &a, &x) == 1 && a == v) {
                s->sid[v] = s->sid[B] = s->sid[C] = -4;
                s->group[v] = s->group[B] = s->group[C] = min3(v, B, C);
                st->n_trim3_hub += 3;
                break;
            }
        }
    }
}

/* coloring_wcc (src/color_propagation.h:468-593): max-label pull over active
 * in- and out-neighbours, then pointer jumping with a depth cap of 100, until
 * a pass changes nothing.  Leaves color[v] = max vertex id of v's WCC. */
static void coloring_wcc(st_t *s)
{
    const oc_graph *g = s->g;
    for (;;) {
        int changed = 0;
        for (int64_t i = 0; i < s->fq; ++i) {
            int64_t v = s->Q[i];
            if (s->sid[v] != ACT) continue;
            for (int dir = 0; dir < 2; ++dir) {
                const int64_t *beg = dir ? g->fw_beg : g->bw_beg;
                const int32_t *adj = dir ? g->fw_adj : g->bw_adj;
                for (int64_t e = beg[v]; e < beg[v + 1]; ++e) {
                    int64_t w = adj[e];
                    if (w == v || s->sid[w] != ACT) continue;
                    if (s->color[v] < s->color[w]) { s->color[v] = s->color[w]; changed = 1; }
                }
            }
        }
        if (!changed) return;
        for (int64_t i = 0; i < s->fq; ++i) {
            int64_t v = s->Q[i];
            if (s->sid[v] != ACT || s->color[v] == v) continue;
            int64_t root = s->color[v];
            int depth = 0;
            while (s->color[root] != root && depth < 100) { root = s->color[root]; depth++; }
            int64_t u = v;
            while (u != root && s->color[u] != root) {
                int64_t prev = u;
                u = s->color[u];
                s->color[prev] = root;
            }
        }
    }
}

static int cmp_i64(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* init_fw_sa (src/fw_bw.h:1548-1583).  FIX(Q3): the reference resets fw_sa at
 * queue *positions* [vert_beg, vert_end) instead of at the queue's vertices,
 * so a stale forward depth equal to a pivot id hides vertices from that
 * pivot's forward search; here the queue's vertices are reset.  The set of
 * distinct WCC colours (a std::set in the reference) is counted. */
static int64_t init_fw_sa(st_t *s)
{
    for (int64_t i = 0; i < s->fq; ++i)
        s->fw_sa[(s->quirks & OC_Q3) ? i : s->Q[i]] = -1;
    if (s->fq == 0) return 0;
    int64_t *c = (int64_t *)malloc((size_t)s->fq * sizeof(int64_t));
    if (!c) return -1;
    for (int64_t i = 0; i < s->fq; ++i) c[i] = s->color[s->Q[i]];
    qsort(c, (size_t)s->fq, sizeof(int64_t), cmp_i64);
    int64_t n = 1;
    for (int64_t i = 1; i < s->fq; ++i) n += c[i] != c[i - 1];
    free(c);
    return n;
}

/* mice_fw_bw (src/fw_bw.h:1585-1691), serial: for each still-unlabelled
 * worklist vertex v in queue order, forward search over active vertices
 * marking fw_sa = v, then backward search inside that set marking the SCC.
 * FIX(Q2): the SCC is keyed by the pivot in group[], and its class code is
 * pivot + 2, so pivots 0 and 1 cannot collide with "unlabelled" or "giant".
 * Uses fw_sa as the per-pivot mark, as the reference does; fw_sa holds int32,
 * which bounds V below 2^31 as the reference's own index_t does. */
static void mice_fw_bw(st_t *s, oc_stats *st)
{
    const oc_graph *g = s->g;
    int64_t *q = s->ring, cap = s->fq > 0 ? s->fq : 1;
    for (int64_t i = 0; i < s->fq; ++i) {
        int64_t v = s->Q[i];
        if (s->sid[v] != ACT) continue;
        int64_t head = 0, tail = 0;
        s->fw_sa[v] = (int32_t)v;
        q[tail++] = v;
        if (tail == cap) tail = 0;
        while (head != tail) {
            int64_t x = q[head++];
            if (head == cap) head = 0;
            for (int64_t e = g->fw_beg[x]; e < g->fw_beg[x + 1]; ++e) {
                int64_t w = g->fw_adj[e];
                if (s->sid[w] == ACT && s->fw_sa[w] != v) {
                    q[tail++] = w;
                    if (tail == cap) tail = 0;
                    s->fw_sa[w] = (int32_t)v;
                }
            }
        }
        int64_t code = (s->quirks & OC_Q2) ? v : v + 2;
        s->sid[v] = code;
        s->group[v] = v;
        int64_t members = 1;
        q[tail++] = v;
        if (tail == cap) tail = 0;
        while (head != tail) {
            int64_t x = q[head++];
            if (head == cap) head = 0;
            for (int64_t e = g->bw_beg[x]; e < g->bw_beg[x + 1]; ++e) {
                int64_t w = g->bw_adj[e];
                if (s->sid[w] == ACT && s->fw_sa[w] == v) {
                    if (code == ACT) {
                        /* Q2 with pivot 0: the member's new code is 0, i.e.
                         * still "unlabelled", so the reference's backward
                         * search (fw_bw.h:1672-1684) re-queues it forever */
                        s->nonterminating = 1;
                        return;
                    }
                    q[tail++] = w;
                    if (tail == cap) tail = 0;
                    s->sid[w] = code;
                    s->group[w] = v;
                    members++;
                }
            }
        }
        st->n_mice_vertices += members;
        st->n_mice_scc++;
    }
}

/* Minimum vertex id per group key (keys are vertex ids in [0, V)). */
static void canon_groups(int64_t V, const int64_t *group, int32_t *labels)
{
    int64_t *mn = (int64_t *)malloc((size_t)(V > 0 ? V : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < V; ++i) mn[i] = INT64_MAX;
    for (int64_t v = 0; v < V; ++v)
        if (v < mn[group[v]]) mn[group[v]] = v;
    for (int64_t v = 0; v < V; ++v) labels[v] = (int32_t)mn[group[v]];
    free(mn);
}

int oc_ispan(const oc_graph *g, int alpha, int beta, int gamma, double theta, int quirks,
             int32_t *labels, int32_t *codes, oc_stats *st)
{
    oc_stats dummy;
    if (!st) st = &dummy;
    memset(st, 0, sizeof(*st));
    st->pivot = -1;
    const int64_t V = g->V;
    const double avg_degree = V ? (double)g->E / (double)V : 0.0;
    size_t n1 = (size_t)(V + 1);
    st_t s;
    memset(&s, 0, sizeof(s));
    s.g = g;
    s.quirks = quirks;
    s.sid = (int64_t *)calloc(n1, sizeof(int64_t));
    s.group = (int64_t *)calloc(n1, sizeof(int64_t));
    s.fw_sa = (int32_t *)malloc(n1 * sizeof(int32_t));
    s.bw_sa = (int32_t *)malloc(n1 * sizeof(int32_t));
    s.color = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.Q = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.tmpq = (int64_t *)malloc(n1 * sizeof(int64_t));
    s.ring = (int64_t *)malloc(n1 * sizeof(int64_t));
    int64_t *fq2 = (int64_t *)malloc(n1 * sizeof(int64_t));
    int64_t *tq2 = (int64_t *)malloc(n1 * sizeof(int64_t));
    int rc = 0;
    if (!s.sid || !s.group || !s.fw_sa || !s.bw_sa || !s.color || !s.Q || !s.tmpq || !s.ring || !fq2 || !tq2) {
        rc = -1;
        goto out;
    }
    /* initialisation (scc_core.cpp:116-125) */
    for (int64_t i = 0; i < V + 1; ++i) {
        s.color[i] = i;
        s.fw_sa[i] = -1;
        s.bw_sa[i] = -1;
        s.sid[i] = 0;
    }
    trim_1_first(&s, st);                    /* scc_core.cpp:177 */
    generate_frontier_queue(&s);             /* scc_core.cpp:353 */
    st->fq_after_trim1 = s.fq;
    int64_t fq_size = s.fq;
    int64_t root = pivot_selection_from_fq(&s); /* scc_core.cpp:382 */
    st->pivot = root;
    if (root >= 0) {
        st->fw_levels = fw_bfs_fq_queue(&s, root, alpha, beta, gamma, avg_degree); /* :447 */
        int64_t ffq = bw_gfq_from_fw(&s, fq2);                                      /* :476 */
        st->fw_size = ffq;
        st->bw_levels = bw_bfs_fq_queue(&s, root, fq2, ffq, alpha, beta, gamma, avg_degree, tq2); /* :507 */
        for (int64_t v = 0; v < V; ++v)
            if (s.sid[v] == 1) { s.group[v] = root; st->giant_size++; }
    }
    /* trim-1 loop, at most TRIM_TIMES=3 passes, theta stop (scc_core.cpp:562-602) */
    {
        int64_t prev = fq_size;
        int times = 0;
        while (prev > 0 && times < 3) {
            trim_1_from_fq_gfq(&s, st);
            fq_size = s.fq;
            if (prev - fq_size < prev * theta) break;
            prev = fq_size;
            times++;
        }
    }
    if (fq_size > 0) { /* scc_core.cpp:609-935 */
        trim_2_from_fq(&s, st);     /* :631 */
        trim_3_1_from_fq(&s, st);   /* :668 */
        trim_3_2_from_fq(&s, st);   /* :697 */
        trim_1_from_fq_gfq(&s, st); /* :757-795, once */
        coloring_wcc(&s);           /* :858 */
        st->n_wcc = init_fw_sa(&s); /* :904 */
        mice_fw_bw(&s, st);         /* :923 */
        if (s.nonterminating) { rc = -2; goto out; }
    }
    canon_groups(V, s.group, labels);
    st->scc_count = oc_count(labels, V);
    if (codes) {
        for (int64_t v = 0; v < V; ++v) codes[v] = (int32_t)s.sid[v];
        codes[V] = 0; /* Q1: the reference reports over V+1 slots */
    }
out:
    free(s.sid); free(s.group); free(s.fw_sa); free(s.bw_sa); free(s.color);
    free(s.Q); free(s.tmpq); free(s.ring); free(fq2); free(tq2);
    return rc;
}

/* ---------------------------------------------------------------------------
 * Iterative Tarjan (independent of iSpan).  Labels = min vertex id per SCC.
 */
int64_t oc_tarjan(const oc_graph *g, const int32_t *key, int32_t *labels)
{
    const int64_t V = g->V;
    if (V == 0) return 0;
    int64_t *idx = (int64_t *)malloc((size_t)V * sizeof(int64_t));
    int64_t *low = (int64_t *)malloc((size_t)V * sizeof(int64_t));
    int64_t *stk = (int64_t *)malloc((size_t)V * sizeof(int64_t));
    int64_t *cs_v = (int64_t *)malloc((size_t)V * sizeof(int64_t));
    int64_t *cs_e = (int64_t *)malloc((size_t)V * sizeof(int64_t));
    unsigned char *on = (unsigned char *)calloc((size_t)V, 1);
    if (!idx || !low || !stk || !cs_v || !cs_e || !on) {
        free(idx); free(low); free(stk); free(cs_v); free(cs_e); free(on);
        return -1;
    }
    for (int64_t i = 0; i < V; ++i) idx[i] = -1;
    int64_t counter = 0, sp = 0, ncomp = 0;
    for (int64_t r = 0; r < V; ++r) {
        if (idx[r] != -1) continue;
        int64_t cp = 0;
        cs_v[cp] = r; cs_e[cp] = g->fw_beg[r]; cp++;
        idx[r] = low[r] = counter++;
        stk[sp++] = r; on[r] = 1;
        while (cp > 0) {
            int64_t v = cs_v[cp - 1];
            int64_t e = cs_e[cp - 1];
            int descended = 0;
            int singleton = key && key[v] == -1;
            int64_t end = singleton ? e : g->fw_beg[v + 1];
            for (; e < end; ++e) {
                int64_t w = g->fw_adj[e];
                if (key && key[w] != key[v]) continue;
                if (idx[w] == -1) {
                    cs_e[cp - 1] = e + 1;
                    idx[w] = low[w] = counter++;
                    stk[sp++] = w; on[w] = 1;
                    cs_v[cp] = w; cs_e[cp] = g->fw_beg[w]; cp++;
                    descended = 1;
                    break;
                } else if (on[w] && idx[w] < low[v]) {
                    low[v] = idx[w];
                }
            }
            if (descended) continue;
            cs_e[cp - 1] = e;
            if (low[v] == idx[v]) {
                int64_t mn = INT64_MAX, k = sp;
                do { --k; if (stk[k] < mn) mn = stk[k]; } while (stk[k] != v);
                while (sp > k) { int64_t w = stk[--sp]; on[w] = 0; labels[w] = (int32_t)mn; }
                ncomp++;
            }
            cp--;
            if (cp > 0) {
                int64_t p = cs_v[cp - 1];
                if (low[v] < low[p]) low[p] = low[v];
            }
        }
    }
    free(idx); free(low); free(stk); free(cs_v); free(cs_e); free(on);
    return ncomp;
}

int64_t oc_count(const int32_t *labels, int64_t V)
{
    int64_t n = 0;
    for (int64_t v = 0; v < V; ++v) n += labels[v] == v;
    return n;
}

int64_t oc_histogram(const int32_t *labels, int64_t V, int64_t *sizes, int64_t *counts, int64_t cap)
{
    if (V == 0) return 0;
    int64_t *sz = (int64_t *)calloc((size_t)V, sizeof(int64_t));
    int64_t *by = (int64_t *)calloc((size_t)V + 1, sizeof(int64_t));
    if (!sz || !by) { free(sz); free(by); return -1; }
    for (int64_t v = 0; v < V; ++v) sz[labels[v]]++;
    for (int64_t v = 0; v < V; ++v)
        if (sz[v]) by[sz[v]]++;
    int64_t n = 0;
    for (int64_t s = 1; s <= V; ++s)
        if (by[s]) {
            if (n < cap) { sizes[n] = s; counts[n] = by[s]; }
            n++;
        }
    free(sz); free(by);
    return n;
}

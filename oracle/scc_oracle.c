/*
 * CPU oracle for the SCC engine -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference algorithm for the SCC path
 * (ShashwaTTrigunayaT/DynamicGraphs_SCC, src/ and gm_graph/).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and only
 * as the checker.  The product library never links or calls anything here.
 *
 * Parity is pinned against the reference itself: oracle/Makefile compiles the
 * reference's own sources (gm_graph/src/*.cc + src/*.cc) into oracle/_ref/, and
 * tests/golden/make_golden.py records that build's method-2 and Tarjan labels
 * on seeded graphs as fixtures; tests/test_oracle.py checks this file against
 * them.
 *
 * Conventions (gm_graph/inc/gm_graph_typedef.h:17-20, src/scc.h:19-22):
 *   node/edge ids are int32; colour -1 = initial, -2 = SCC found, >= 0 fresh;
 *   scc[v] is the representative vertex of v's SCC.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define COLOR_INIT (-1)
#define COLOR_DONE (-2)

/* ------------------------------------------------------------------------ */
/* CSR construction: gm_graph::freeze + do_semi_sort + make_reverse_edges     */
/* (gm_graph/src/gm_graph.cc:60-101, 385-420, 193-287).  Adjacency lists are   */
/* sorted by destination, the transpose by source; duplicates and self-loops   */
/* are kept exactly as the reference keeps them.                               */
/* ------------------------------------------------------------------------ */
static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* One side: rows = key, columns = val, each row sorted.  Two stable counting
 * passes (by val, then by key) give rows already sorted, no comparison sort. */
static void csr_side(int32_t n, int64_t m, const int32_t* key, const int32_t* val, int32_t* off, int32_t* out) {
    int32_t* cnt = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int64_t* tmp_pos = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
    int64_t* vstart = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t e = 0; e < m; ++e) vstart[val[e] + 1]++;
    for (int32_t v = 0; v < n; ++v) vstart[v + 1] += vstart[v];
    for (int64_t e = 0; e < m; ++e) tmp_pos[vstart[val[e]]++] = e;   /* edges ordered by val */
    memset(off, 0, sizeof(int32_t) * ((size_t)n + 1));
    for (int64_t e = 0; e < m; ++e) off[key[e] + 1]++;
    for (int32_t v = 0; v < n; ++v) off[v + 1] += off[v];
    memcpy(cnt, off, sizeof(int32_t) * ((size_t)n + 1));
    for (int64_t i = 0; i < m; ++i) { int64_t e = tmp_pos[i]; order[cnt[key[e]]++] = e; }
    for (int64_t i = 0; i < m; ++i) out[i] = val[order[i]];
    free(cnt); free(tmp_pos); free(order); free(vstart);
}

void orc_build_csr(int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                   int32_t* begin, int32_t* node_idx, int32_t* r_begin, int32_t* r_node_idx) {
    csr_side(n, m, src, dst, begin, node_idx);
    csr_side(n, m, dst, src, r_begin, r_node_idx);
}

/* Generator post-processing: drop self-loops and duplicate edges (in place),
 * returning the new edge count.  Sorting by (src, dst) via csr_side. */
int64_t orc_dedup_edges(int32_t n, int64_t m, int32_t* src, int32_t* dst) {
    int32_t* off = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    int32_t* adj = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    csr_side(n, m, src, dst, off, adj);
    int64_t k = 0;
    for (int32_t v = 0; v < n; ++v) {
        int32_t prev = -1;
        for (int32_t i = off[v]; i < off[v + 1]; ++i) {
            int32_t w = adj[i];
            if (w == v || w == prev) continue;
            prev = w;
            src[k] = v; dst[k] = w; k++;
        }
    }
    free(off); free(adj);
    (void)cmp_i32;
    return k;
}

/* ------------------------------------------------------------------------ */
/* Tarjan, iterative form of scc_tarjan_recurse / do_tarjan_all               */
/* (src/scc_tarjan.cc:99-149).  scc[w] = v, the root of w's SCC in the DFS.    */
/* Vertices whose colour is already -2 are skipped as in do_tarjan_all:145.    */
/* ------------------------------------------------------------------------ */
void orc_tarjan(int32_t n, const int32_t* begin, const int32_t* node_idx, int32_t* scc) {
    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* low = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    uint8_t* onstk = (uint8_t*)calloc((size_t)n, 1);
    int32_t* stk = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* cs_v = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);  /* call stack: vertex */
    int32_t* cs_e = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);  /* call stack: next edge */
    int32_t counter = 0, sp = 0;
    for (int32_t v = 0; v < n; ++v) { idx[v] = -1; scc[v] = -1; }
    for (int32_t s = 0; s < n; ++s) {
        if (idx[s] >= 0) continue;
        int32_t csp = 0;
        cs_v[csp] = s; cs_e[csp] = begin[s]; csp++;
        idx[s] = low[s] = counter++; stk[sp++] = s; onstk[s] = 1;
        while (csp > 0) {
            int32_t v = cs_v[csp - 1];
            int32_t e = cs_e[csp - 1];
            if (e < begin[v + 1]) {
                cs_e[csp - 1] = e + 1;
                int32_t w = node_idx[e];
                if (idx[w] < 0) {
                    idx[w] = low[w] = counter++; stk[sp++] = w; onstk[w] = 1;
                    cs_v[csp] = w; cs_e[csp] = begin[w]; csp++;
                } else if (onstk[w] && idx[w] < low[v]) {
                    low[v] = idx[w];
                }
            } else {
                csp--;
                if (low[v] == idx[v]) {
                    int32_t w;
                    do { w = stk[--sp]; onstk[w] = 0; scc[w] = v; } while (w != v);
                }
                if (csp > 0) {
                    int32_t p = cs_v[csp - 1];
                    if (low[v] < low[p]) low[p] = low[v];
                }
            }
        }
    }
    free(idx); free(low); free(onstk); free(stk); free(cs_v); free(cs_e);
}

/* Canonical relabelling: component id = smallest member vertex id. */
void orc_canonical(int32_t n, const int32_t* scc, int32_t* out) {
    int32_t* minm = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int32_t v = 0; v < n; ++v) minm[v] = INT32_MAX;
    for (int32_t v = 0; v < n; ++v) { int32_t r = scc[v]; if (r >= 0 && v < minm[r]) minm[r] = v; }
    for (int32_t v = 0; v < n; ++v) out[v] = (scc[v] >= 0) ? minm[scc[v]] : -1;
    free(minm);
}

/* ------------------------------------------------------------------------ */
/* Trim1 to its fixpoint: trim_once_node (src/scc_trim1.cc:38-110) repeated    */
/* until nothing changes (the CUDA reference's TRIM_STOP=0 form).  A vertex of */
/* colour c is trimmed (colour -2, scc = itself) when it has no out-neighbour  */
/* or no in-neighbour of colour c other than itself.  The fixpoint set is      */
/* unique, so it does not depend on visiting order.  Returns #trimmed.         */
/* ------------------------------------------------------------------------ */
static int has_live_nbr(const int32_t* b, const int32_t* a, const int32_t* color, int32_t v, int32_t c) {
    for (int32_t k = b[v]; k < b[v + 1]; ++k) {
        int32_t w = a[k];
        if (w != v && color[w] == c) return 1;
    }
    return 0;
}

int64_t orc_trim1_fixpoint(int32_t n, const int32_t* begin, const int32_t* node_idx,
                           const int32_t* r_begin, const int32_t* r_node_idx,
                           int32_t* color, int32_t* scc) {
    /* worklist peel: check every vertex once, re-check neighbours of trimmed ones */
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    uint8_t* inq = (uint8_t*)calloc((size_t)n, 1);
    int64_t head = 0, tail = 0, cap = n + 1, count = 0;
    for (int32_t v = 0; v < n; ++v) if (color[v] != COLOR_DONE) { q[tail] = v; tail = (tail + 1) % cap; inq[v] = 1; }
    while (head != tail) {
        int32_t v = q[head]; head = (head + 1) % cap; inq[v] = 0;
        int32_t c = color[v];
        if (c == COLOR_DONE) continue;
        if (has_live_nbr(begin, node_idx, color, v, c) && has_live_nbr(r_begin, r_node_idx, color, v, c)) continue;
        color[v] = COLOR_DONE; scc[v] = v; count++;
        for (int pass = 0; pass < 2; ++pass) {
            const int32_t* b = pass ? r_begin : begin;
            const int32_t* a = pass ? r_node_idx : node_idx;
            for (int32_t k = b[v]; k < b[v + 1]; ++k) {
                int32_t w = a[k];
                if (color[w] == c && !inq[w]) { q[tail] = w; tail = (tail + 1) % cap; inq[w] = 1; }
            }
        }
    }
    free(q); free(inq);
    return count;
}

/* ------------------------------------------------------------------------ */
/* Trim2 (src/scc_trim2_new.cc:3-102): {n,k} with n<k is a 2-vertex SCC when   */
/* n's only live out-neighbour (ignoring self-loops and repeats) is k and k's  */
/* is n, or the same through in-edges.  Restated with every decision taken on  */
/* the colours as they stood before the pass (such pairs are disjoint), so the */
/* result is unique.  Returns #vertices trimmed.                               */
/* ------------------------------------------------------------------------ */
static int degree_is_one(const int32_t* b, const int32_t* a, const int32_t* color, int32_t c, int32_t v, int32_t* nbr) {
    int32_t the = -1; int cnt = 0;
    for (int32_t k = b[v]; k < b[v + 1]; ++k) {
        int32_t w = a[k];
        if (w == v || w == the || color[w] != c) continue;
        cnt++; the = w;
        if (cnt == 2) return 0;
    }
    *nbr = the;
    return cnt == 1;
}

int64_t orc_trim2(int32_t n, const int32_t* begin, const int32_t* node_idx,
                  const int32_t* r_begin, const int32_t* r_node_idx, int32_t* color, int32_t* scc) {
    int32_t* mate = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int64_t count = 0;
    for (int32_t v = 0; v < n; ++v) {
        mate[v] = -1;
        int32_t c = color[v];
        if (c == COLOR_DONE) continue;
        int32_t k, kk;
        if (degree_is_one(begin, node_idx, color, c, v, &k) && v < k &&
            degree_is_one(begin, node_idx, color, c, k, &kk) && kk == v) { mate[v] = k; continue; }
        if (degree_is_one(r_begin, r_node_idx, color, c, v, &k) && v < k &&
            degree_is_one(r_begin, r_node_idx, color, c, k, &kk) && kk == v) { mate[v] = k; continue; }
    }
    for (int32_t v = 0; v < n; ++v) {
        int32_t k = mate[v];
        if (k < 0) continue;
        color[v] = color[k] = COLOR_DONE;
        scc[v] = scc[k] = v;
        count += 2;
    }
    free(mate);
    return count;
}

/* ------------------------------------------------------------------------ */
/* Min-reach colouring, the fixpoint of propagate_color (src/scc_weak.cc:     */
/* 65-125) with the initial labels of do_global_wcc (scc_weak.cc:137-149):    */
/* raw(t) = t, or t | 0x20000000 when t's out-degree is >= 50.  wcc[v] ends as */
/* the minimum raw value over the live vertices of v's colour reachable from  */
/* v.  Computed exactly by backward searches from raw values in increasing    */
/* order.  Vertices of colour -2 get -1.                                       */
/* ------------------------------------------------------------------------ */
typedef struct { int32_t raw; int32_t v; } raw_pair;
static int cmp_raw(const void* a, const void* b) {
    int32_t x = ((const raw_pair*)a)->raw, y = ((const raw_pair*)b)->raw;
    return (x > y) - (x < y);
}

void orc_wcc_minreach(int32_t n, const int32_t* begin, const int32_t* r_begin, const int32_t* r_node_idx,
                      const int32_t* color, int32_t* wcc) {
    raw_pair* order = (raw_pair*)malloc(sizeof(raw_pair) * (size_t)(n > 0 ? n : 1));
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t cnt = 0;
    for (int32_t v = 0; v < n; ++v) {
        wcc[v] = -1;
        if (color[v] == COLOR_DONE) continue;
        int32_t raw = (begin[v + 1] - begin[v] >= 50) ? (v | 0x20000000) : v;
        order[cnt].raw = raw; order[cnt].v = v; cnt++;
    }
    qsort(order, (size_t)cnt, sizeof(raw_pair), cmp_raw);
    for (int32_t i = 0; i < cnt; ++i) {
        int32_t r = order[i].v;
        if (wcc[r] >= 0) continue;
        int32_t c = color[r], h = 0, t = 0;
        wcc[r] = order[i].raw; q[t++] = r;
        while (h < t) {
            int32_t x = q[h++];
            for (int32_t k = r_begin[x]; k < r_begin[x + 1]; ++k) {
                int32_t u = r_node_idx[k];
                if (color[u] == c && wcc[u] < 0) { wcc[u] = order[i].raw; q[t++] = u; }
            }
        }
    }
    free(order); free(q);
}

/* Forward reachability from `pivot` over vertices of colour `c` (the navigator
 * of fw_trim_global, src/scc_fb_global.cc:32-69); marks reached[v] = 1. */
int64_t orc_reach(int32_t n, const int32_t* b, const int32_t* a, const int32_t* color, int32_t c,
                  int32_t pivot, uint8_t* reached) {
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    int32_t h = 0, t = 0;
    memset(reached, 0, (size_t)n);
    reached[pivot] = 1; q[t++] = pivot;
    while (h < t) {
        int32_t x = q[h++];
        for (int32_t k = b[x]; k < b[x + 1]; ++k) {
            int32_t w = a[k];
            if (!reached[w] && color[w] == c) { reached[w] = 1; q[t++] = w; }
        }
    }
    free(q);
    return t;
}

/* ------------------------------------------------------------------------ */
/* Global FW-BW (do_fw_bw_global_main, src/scc_fb_global.cc:133-219) from a   */
/* given pivot of colour `base`: FW set gets fw_color, the intersection with   */
/* the BW set becomes an SCC (scc = pivot, colour -2), the rest of the BW set  */
/* gets bw_color.  Returns the SCC size; *fw_out/*bw_out get the set sizes     */
/* net of the SCC, as the reference's counters report them.                    */
/* ------------------------------------------------------------------------ */
int64_t orc_fw_bw(int32_t n, const int32_t* begin, const int32_t* node_idx,
                  const int32_t* r_begin, const int32_t* r_node_idx,
                  int32_t* color, int32_t* scc, int32_t base, int32_t pivot,
                  int32_t fw_color, int32_t bw_color, int64_t* fw_out, int64_t* bw_out) {
    uint8_t* fw = (uint8_t*)malloc((size_t)(n > 0 ? n : 1));
    uint8_t* bw = (uint8_t*)malloc((size_t)(n > 0 ? n : 1));
    orc_reach(n, begin, node_idx, color, base, pivot, fw);
    orc_reach(n, r_begin, r_node_idx, color, base, pivot, bw);
    int64_t s = 0, f = 0, w = 0;
    for (int32_t v = 0; v < n; ++v) {
        if (color[v] != base) continue;
        if (fw[v] && bw[v]) { color[v] = COLOR_DONE; scc[v] = pivot; s++; }
        else if (fw[v]) { color[v] = fw_color; f++; }
        else if (bw[v]) { color[v] = bw_color; w++; }
    }
    if (fw_out) *fw_out = f;
    if (bw_out) *bw_out = w;
    free(fw); free(bw);
    return s;
}

/* Pivot rule of this engine (the reference picks the first vertex of the
 * colour, src/scc_color.cc:64-93; the B200 engine picks the vertex of the
 * colour with the largest in-degree x out-degree, ties broken by a fixed
 * hash of the id).  Restated so phase-level outputs can be compared. */
static uint32_t pivot_hash(uint32_t v) {
    uint32_t x = v * 0x9E3779B1u;
    x ^= x >> 16; x *= 0x85EBCA6Bu; x ^= x >> 13;
    return x;
}
uint64_t orc_pivot_key(const int32_t* begin, const int32_t* r_begin, int32_t v) {
    uint64_t prod = (uint64_t)(uint32_t)(begin[v + 1] - begin[v]) * (uint64_t)(uint32_t)(r_begin[v + 1] - r_begin[v]);
    if (prod > 0xFFFFFFFFull) prod = 0xFFFFFFFFull;
    return (prod << 32) | pivot_hash((uint32_t)v);
}
int32_t orc_choose_pivot(int32_t n, const int32_t* begin, const int32_t* r_begin, const int32_t* color, int32_t c) {
    int32_t best = -1; uint64_t bk = 0;
    for (int32_t v = 0; v < n; ++v) {
        if (color[v] != c) continue;
        uint64_t k = orc_pivot_key(begin, r_begin, v);
        if (best < 0 || k > bk) { best = v; bk = k; }
    }
    return best;
}

/* Full SCC decomposition by Tarjan followed by canonical relabelling. */
void orc_scc_canonical(int32_t n, const int32_t* begin, const int32_t* node_idx, int32_t* out) {
    int32_t* scc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    orc_tarjan(n, begin, node_idx, scc);
    orc_canonical(n, scc, out);
    free(scc);
}

/* ------------------------------------------------------------------------ */
/* Method 7: topological levels of the condensation graph and the levels an   */
/* inserted batch affects (create_scc_edges + BFS, src/common_main.h:85-108,   */
/* 180-262).  Restated literally: a FIFO queue seeded, in id order, with the   */
/* nodes that have no in-edge but some out-edge; every edge of a processed    */
/* node decrements its child's in-degree (duplicates counted), queues the      */
/* child at zero, and overwrites the child's level with the parent's + 1.      */
/* ------------------------------------------------------------------------ */
int32_t orc_topo_levels(int32_t n, const int32_t* begin, const int32_t* adj, int32_t* level) {
    int32_t* indeg = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    int32_t* queue = (int32_t*)malloc(sizeof(int32_t) * ((size_t)n + 1));
    int64_t head = 0, tail = 0;
    int32_t max_level = 0;
    for (int32_t v = 0; v < n; ++v) level[v] = 0;
    for (int64_t k = 0; k < begin[n]; ++k) indeg[adj[k]]++;
    for (int32_t v = 0; v < n; ++v)
        if (indeg[v] == 0 && begin[v + 1] > begin[v]) queue[tail++] = v;
    while (head < tail) {
        int32_t top = queue[head++];
        for (int32_t k = begin[top]; k < begin[top + 1]; ++k) {
            int32_t c = adj[k];
            if (--indeg[c] == 0) queue[tail++] = c;
            level[c] = level[top] + 1;
            if (level[c] > max_level) max_level = level[c];
        }
    }
    free(indeg);
    free(queue);
    return max_level;
}

/* affect_level: +1 at min(level), -1 at max(level) + 1 for every inserted edge
 * whose endpoints lie in different SCCs, then the inclusive prefix sum
 * (parallel_prefix_sum, common_main.h:109-148, here in exact integers).
 * affected[0..max_level]; returns the count of zero entries (unaffected). */
int32_t orc_affected_levels(const int32_t* label, const int32_t* level, int32_t max_level, int64_t k,
                            const int32_t* src, const int32_t* dst, int32_t* affected) {
    int32_t* diff = (int32_t*)calloc((size_t)max_level + 2, sizeof(int32_t));
    for (int64_t i = 0; i < k; ++i) {
        int32_t a = label[src[i]], b = label[dst[i]];
        if (a == b) continue;
        int32_t la = level[a], lb = level[b];
        diff[la < lb ? la : lb] += 1;
        diff[(la > lb ? la : lb) + 1] -= 1;
    }
    int32_t run = 0, zeros = 0;
    for (int32_t l = 0; l <= max_level; ++l) {
        run += diff[l];
        affected[l] = run;
        zeros += run == 0;
    }
    free(diff);
    return zeros;
}

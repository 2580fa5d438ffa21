/*
 * oracle.c - TEST INFRASTRUCTURE ONLY.  A plain-C restatement of the
 * reference's CPU adjacency-list algorithms (GraphHET include/CPU_adj_list/)
 * over CSR arrays, used by the tests and by bench.py's CPU baseline as the
 * checker.  Nothing in the product (graphhet_b200/, include/) calls it.
 *
 * Parity is pinned twice: against outputs of the reference's own CPU code
 * compiled from its sources (oracle/_ref, built by oracle/Makefile), and
 * against the known answers committed under tests/golden/.
 *
 * Graph arguments are CSR arrays: rowptr[n+1], col[m] (rows sorted), w[m].
 * The reference's graph_structure keeps the same data as sorted
 * vector<pair<int,double>> rows (CPU_adj_list.hpp:16-70).
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/ghb_gen.h"

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------ generators */
/* The seeded inputs of include/ghb_gen.h, restated on the CPU. */

ORC_API void orc_gen_rmat(int scale, int64_t n_edges, uint64_t seed, double a, double b, double c,
                          int permute, int32_t* src, int32_t* dst) {
    ghb_rmat_thresholds t = ghb_rmat_make_thresholds(a, b, c);
    ghb_perm perm = ghb_perm_make(seed, scale);
    uint64_t stream = ghb_stream(seed, GHB_PURPOSE_RMAT);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_edges; ++e) {
        uint32_t u, v;
        ghb_rmat_edge(stream, t, scale, (uint64_t)e, &u, &v);
        if (permute) {
            u = ghb_perm_apply(&perm, u);
            v = ghb_perm_apply(&perm, v);
        }
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
    }
}

ORC_API void orc_gen_grid(int32_t rows, int32_t cols, int32_t* src, int32_t* dst) {
    int64_t right = (int64_t)rows * (cols - 1), down = (int64_t)(rows - 1) * cols;
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < right + down; ++e) {
        int64_t u, v;
        if (e < right) {
            int64_t r = e / (cols - 1), c = e % (cols - 1);
            u = r * cols + c;
            v = u + 1;
        } else {
            u = e - right;
            v = u + cols;
        }
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
    }
}

ORC_API void orc_gen_er(int32_t n, int64_t n_edges, uint64_t seed, int32_t* src, int32_t* dst) {
    uint64_t stream = ghb_stream(seed, GHB_PURPOSE_ER);
#pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < n_edges; ++e) {
        uint32_t u, v;
        ghb_er_edge(stream, (uint32_t)n, (uint64_t)e, &u, &v);
        src[e] = (int32_t)u;
        dst[e] = (int32_t)v;
    }
}

/* keep[e] = 0 when src[e] is a dangling vertex of the seed (ghb_is_dangling). */
ORC_API void orc_gen_dangling_keep(int64_t n_edges, const int32_t* src, uint64_t seed, double fraction,
                                   uint8_t* keep) {
    const uint32_t threshold = fraction >= 1.0 ? 0xffffffffu : (uint32_t)(fraction * 4294967296.0);
    const uint64_t ds = ghb_stream(seed, GHB_PURPOSE_DANGLING);
    for (int64_t e = 0; e < n_edges; ++e) keep[e] = ghb_is_dangling(ds, (uint32_t)src[e], threshold) ? 0 : 1;
}

ORC_API double orc_pair_weight(uint64_t seed, int32_t u, int32_t v, int mode) {
    return ghb_pair_weight(ghb_stream(seed, GHB_PURPOSE_WEIGHT), (uint32_t)u, (uint32_t)v, mode);
}

/* ------------------------------------------------------------ CSR builder */
/* Same contract as ghb_csr_build: duplicates merged (graph_structure keeps
 * one entry per pair, sorted_vector_binary_operations.hpp:89-101; the last
 * add_edge wins the weight), optional symmetrisation (ldbc.hpp:240-242),
 * optional self-loop removal, optional transpose.  Returns m or -1 on a bad
 * endpoint. */
typedef struct {
    int32_t c;
    uint32_t idx;
} orc_entry;

static int cmp_entry(const void* a, const void* b) {
    const orc_entry* x = (const orc_entry*)a;
    const orc_entry* y = (const orc_entry*)b;
    if (x->c != y->c) return x->c < y->c ? -1 : 1;
    if (x->idx != y->idx) return x->idx < y->idx ? -1 : 1;
    return 0;
}

ORC_API int64_t orc_csr_build(int32_t n, const int32_t* src, const int32_t* dst, const double* w_in,
                              int64_t n_edges, int flags, int weight_mode, uint64_t weight_seed,
                              int32_t* rowptr, int32_t* col, double* w) {
    const int sym = flags & 1, drop = flags & 2, tr = flags & 4;
    for (int64_t i = 0; i < n_edges; ++i)
        if (src[i] < 0 || src[i] >= n || dst[i] < 0 || dst[i] >= n) return -1;
    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_edges; ++i) {
        int32_t u = src[i], v = dst[i];
        if (tr) { int32_t t = u; u = v; v = t; }
        if (drop && u == v) continue;
        __atomic_fetch_add(&cnt[u], 1, __ATOMIC_RELAXED);
        if (sym) __atomic_fetch_add(&cnt[v], 1, __ATOMIC_RELAXED);
    }
    int64_t* start = (int64_t*)malloc(((size_t)n + 1) * sizeof(int64_t));
    start[0] = 0;
    for (int32_t r = 0; r < n; ++r) start[r + 1] = start[r] + cnt[r];
    const int64_t total = start[n];
    orc_entry* ent = (orc_entry*)malloc((size_t)(total > 0 ? total : 1) * sizeof(orc_entry));
    int64_t* cur = cnt; /* reuse as cursor */
    for (int32_t r = 0; r <= n; ++r) cur[r] = start[r];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_edges; ++i) {
        int32_t u = src[i], v = dst[i];
        if (tr) { int32_t t = u; u = v; v = t; }
        if (drop && u == v) continue;
        int64_t p = __atomic_fetch_add(&cur[u], 1, __ATOMIC_RELAXED);
        ent[p].c = v;
        ent[p].idx = (uint32_t)i;
        if (sym) {
            int64_t q = __atomic_fetch_add(&cur[v], 1, __ATOMIC_RELAXED);
            ent[q].c = u;
            ent[q].idx = (uint32_t)i;
        }
    }
    /* Sort each row by (column, input index); keep the last of each column. */
    int32_t* kept = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t r = 0; r < n; ++r) {
        orc_entry* row = ent + start[r];
        int64_t len = start[r + 1] - start[r];
        if (len > 1) qsort(row, (size_t)len, sizeof(orc_entry), cmp_entry);
        int64_t k = 0;
        for (int64_t j = 0; j < len; ++j) {
            if (j + 1 < len && row[j + 1].c == row[j].c) continue;
            row[k++] = row[j];
        }
        kept[r] = (int32_t)k;
    }
    rowptr[0] = 0;
    for (int32_t r = 0; r < n; ++r) rowptr[r + 1] = rowptr[r] + kept[r];
    const uint64_t ws = ghb_stream(weight_seed, GHB_PURPOSE_WEIGHT);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t r = 0; r < n; ++r) {
        const orc_entry* row = ent + start[r];
        int32_t o = rowptr[r];
        for (int32_t k = 0; k < kept[r]; ++k) {
            col[o + k] = row[k].c;
            if (w) {
                if (w_in) w[o + k] = w_in[row[k].idx];
                else if (weight_mode) {
                    uint32_t a = tr ? (uint32_t)row[k].c : (uint32_t)r;
                    uint32_t b = tr ? (uint32_t)r : (uint32_t)row[k].c;
                    w[o + k] = ghb_pair_weight(ws, a, b, weight_mode);
                }
            }
        }
    }
    int64_t m = rowptr[n];
    free(kept);
    free(ent);
    free(start);
    free(cnt);
    return m;
}

/* ------------------------------------------------------------------- BFS */
/* CPU_BFS.hpp:10-41: FIFO queue; a vertex at depth d expands only when
 * d + 1 <= max_depth; unreached = INT_MAX. */
ORC_API void orc_bfs(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t root, int32_t max_depth,
                     int32_t* depth) {
    int32_t* q = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    for (int32_t i = 0; i < n; ++i) depth[i] = INT_MAX;
    depth[root] = 0;
    int64_t head = 0, tail = 0;
    q[tail++] = root;
    while (head < tail) {
        int32_t v = q[head++];
        if ((int64_t)depth[v] + 1 <= max_depth) {
            for (int32_t j = rowptr[v]; j < rowptr[v + 1]; ++j) {
                int32_t a = col[j];
                if (depth[a] > depth[v] + 1) {
                    depth[a] = depth[v] + 1;
                    q[tail++] = a;
                }
            }
        }
    }
    free(q);
}

/* ------------------------------------------------------------------ SSSP */
/* CPU_shortest_paths.hpp:19-64: Dijkstra with a binary min-heap of
 * (distance, vertex), lazy deletion, initial distance DBL_MAX; relax when
 * dist[v] > dist[u] + w. */
typedef struct {
    double d;
    int32_t u;
} orc_node;

static void heap_push(orc_node** h, int64_t* size, int64_t* cap, orc_node x) {
    if (*size == *cap) {
        *cap = *cap ? *cap * 2 : 1024;
        *h = (orc_node*)realloc(*h, (size_t)*cap * sizeof(orc_node));
    }
    int64_t i = (*size)++;
    orc_node* a = *h;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (a[p].d <= x.d) break;
        a[i] = a[p];
        i = p;
    }
    a[i] = x;
}

static orc_node heap_pop(orc_node* a, int64_t* size) {
    orc_node top = a[0];
    orc_node x = a[--(*size)];
    int64_t i = 0, s = *size;
    while (1) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        double md = x.d;
        if (l < s && a[l].d < md) { m = l; md = a[l].d; }
        if (r < s && a[r].d < md) { m = r; }
        if (m == i) break;
        a[i] = a[m];
        i = m;
    }
    if (s > 0) a[i] = x;
    return top;
}

ORC_API void orc_sssp(int32_t n, const int32_t* rowptr, const int32_t* col, const double* w, int32_t src,
                      double* dist) {
    for (int32_t i = 0; i < n; ++i) dist[i] = 1.7976931348623157e308; /* DBL_MAX */
    if (src < 0 || src >= n) return;
    dist[src] = 0.0;
    char* vis = (char*)calloc((size_t)n, 1);
    orc_node* h = NULL;
    int64_t size = 0, cap = 0;
    orc_node s0 = {0.0, src};
    heap_push(&h, &size, &cap, s0);
    while (size > 0) {
        int32_t u = heap_pop(h, &size).u;
        if (vis[u]) continue;
        vis[u] = 1;
        for (int32_t j = rowptr[u]; j < rowptr[u + 1]; ++j) {
            int32_t v = col[j];
            double nd = dist[u] + w[j];
            if (dist[v] > nd) {
                dist[v] = nd;
                orc_node x = {nd, v};
                heap_push(&h, &size, &cap, x);
            }
        }
    }
    free(h);
    free(vis);
}

/* ------------------------------------------------------------------- WCC */
/* CPU_connected_components.hpp:12-66, single-threaded: repeat { for every
 * entry (u, v): if the larger of comp[u], comp[v] is a root, hook it under
 * the smaller; then compress every vertex to its root } until no hook.  The
 * fixpoint labels every vertex with the smallest id of its component. */
ORC_API void orc_wcc(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* comp) {
    for (int32_t u = 0; u < n; ++u) comp[u] = u;
    int change = 1;
    while (change) {
        change = 0;
        for (int32_t u = 0; u < n; ++u) {
            for (int32_t j = rowptr[u]; j < rowptr[u + 1]; ++j) {
                int32_t v = col[j];
                int32_t cu = comp[u], cv = comp[v];
                if (cu == cv) continue;
                int32_t hi = cu > cv ? cu : cv, lo = cu + (cv - hi);
                if (hi == comp[hi]) {
                    change = 1;
                    comp[hi] = lo;
                }
            }
        }
        for (int32_t u = 0; u < n; ++u)
            while (comp[u] != comp[comp[u]]) comp[u] = comp[comp[u]];
    }
}

/* -------------------------------------------------------------- PageRank */
/* CPU_PageRank.hpp:12-56: rank = 1/N; per iteration sink_sum over vertices
 * with no out-edges (index order), common = sink_sum*d/N + (1-d)/N,
 * new[v] = common + d * sum_{u in in(v)} rank[u] / outdeg(u) (in-row order). */
ORC_API void orc_pagerank(int32_t n, const int32_t* in_rp, const int32_t* in_col, const int32_t* out_rp,
                          double damp, int32_t iters, double* rank) {
    double* nr = (double*)malloc((size_t)n * sizeof(double));
    for (int32_t i = 0; i < n; ++i) rank[i] = 1 / (double)n;
    const double teleport = (1 - damp) / n;
    for (int32_t it = 0; it < iters; ++it) {
        double sink_sum = 0;
        for (int32_t i = 0; i < n; ++i)
            if (out_rp[i + 1] == out_rp[i]) sink_sum += rank[i];
        const double common = (sink_sum * damp / n) + teleport;
#pragma omp parallel for schedule(dynamic, 4096)
        for (int32_t v = 0; v < n; ++v) {
            double s = 0;
            for (int32_t j = in_rp[v]; j < in_rp[v + 1]; ++j) {
                int32_t u = in_col[j];
                s += rank[u] / (double)(out_rp[u + 1] - out_rp[u]);
            }
            nr[v] = common + damp * s;
        }
        memcpy(rank, nr, (size_t)n * sizeof(double));
    }
    free(nr);
}

/* ------------------------------------------------------------------ CDLP */
/* CPU_Community_Detection.hpp:12-64: labels start as ids; each iteration
 * counts the labels over the in-row then the out-row of v; the new label is
 * the most frequent, the smallest on ties; an isolated vertex keeps its
 * label.  Counting through a sorted buffer gives the same (label, count)
 * table as the reference's unordered_map. */
static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return x < y ? -1 : (x > y);
}

ORC_API void orc_cdlp(int32_t n, const int32_t* in_rp, const int32_t* in_col, const int32_t* out_rp,
                      const int32_t* out_col, int32_t iters, int32_t* label) {
    int32_t* nl = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    for (int32_t i = 0; i < n; ++i) label[i] = i;
    for (int32_t it = 0; it < iters; ++it) {
#pragma omp parallel
        {
            int64_t cap = 1024;
            int32_t* buf = (int32_t*)malloc((size_t)cap * sizeof(int32_t));
#pragma omp for schedule(dynamic, 1024)
            for (int32_t i = 0; i < n; ++i) {
                int64_t len = (int64_t)(in_rp[i + 1] - in_rp[i]) + (out_rp[i + 1] - out_rp[i]);
                if (len == 0) {
                    nl[i] = label[i];
                    continue;
                }
                if (len > cap) {
                    cap = len;
                    buf = (int32_t*)realloc(buf, (size_t)cap * sizeof(int32_t));
                }
                int64_t k = 0;
                for (int32_t j = in_rp[i]; j < in_rp[i + 1]; ++j) buf[k++] = label[in_col[j]];
                for (int32_t j = out_rp[i]; j < out_rp[i + 1]; ++j) buf[k++] = label[out_col[j]];
                qsort(buf, (size_t)len, sizeof(int32_t), cmp_i32);
                int32_t best = buf[0];
                int64_t best_c = 0, run = 0;
                for (int64_t j = 0; j < len; ++j) {
                    run = (j > 0 && buf[j] == buf[j - 1]) ? run + 1 : 1;
                    if (run > best_c) {
                        best_c = run;
                        best = buf[j];
                    }
                }
                nl[i] = best;
            }
            free(buf);
        }
        memcpy(label, nl, (size_t)n * sizeof(int32_t));
    }
    free(nl);
}

/* -------------------------------------------------------------------- TC */
/* CPU_TC.hpp:31-60: for every entry u->v, merge row(u) with row(v); every
 * common w adds 1 to u, v and w.  int32 counters (wrapping, like the
 * reference's `int`). */
ORC_API void orc_tc(int32_t n, const int32_t* rowptr, const int32_t* col, int32_t* counts) {
    uint32_t* c = (uint32_t*)calloc((size_t)n, sizeof(uint32_t));
    for (int32_t u = 0; u < n; ++u) {
        for (int32_t e = rowptr[u]; e < rowptr[u + 1]; ++e) {
            int32_t v = col[e];
            int32_t i = rowptr[u], ie = rowptr[u + 1], j = rowptr[v], je = rowptr[v + 1];
            while (i < ie && j < je) {
                int32_t a = col[i], b = col[j];
                if (a == b) {
                    c[u]++;
                    c[v]++;
                    c[a]++;
                    ++i;
                    ++j;
                } else if (a < b) {
                    ++i;
                } else {
                    ++j;
                }
            }
        }
    }
    for (int32_t u = 0; u < n; ++u) counts[u] = (int32_t)c[u];
    free(c);
}

/* ----------------------------------------------------- TC, oriented (CPU) */
/* Per-vertex triangle incidences of a symmetric, loop-free CSR without
 * repeated entries, by degree orientation: counts[x] = 6 * (triangles that
 * contain x), which is what Tri_Counting (CPU_TC.hpp:31-60) computes on such
 * a graph before its int32 wrap.  It exists because the reference's merge
 * over every entry is quadratic in the hub degrees and does not finish on
 * the benchmark graphs; the tests pin it to orc_tc and to the compiled
 * reference on graphs where those finish.  Returns the triangle count.
 *
 * Orientation: x -> y when (deg x, x) < (deg y, y).  Each triangle is found
 * once, from its lowest corner x, as v in N+(x) and w in N+(x) and N+(v)
 * (a thread-local bitmap marks N+(x)); its three corners are counted in the
 * thread's own counter array, and the arrays are summed at the end. */
ORC_API int64_t orc_tc_oriented(int32_t n, const int32_t* rowptr, const int32_t* col, int64_t* counts) {
    int64_t* pp = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
#define ORC_BEFORE(a, b) ((rowptr[(a) + 1] - rowptr[(a)]) < (rowptr[(b) + 1] - rowptr[(b)]) || \
                          ((rowptr[(a) + 1] - rowptr[(a)]) == (rowptr[(b) + 1] - rowptr[(b)]) && (a) < (b)))
#pragma omp parallel for schedule(dynamic, 4096)
    for (int32_t x = 0; x < n; ++x) {
        int64_t p = 0;
        for (int32_t j = rowptr[x]; j < rowptr[x + 1]; ++j)
            if (ORC_BEFORE(x, col[j])) ++p;
        pp[x + 1] = p;
    }
    for (int32_t x = 0; x < n; ++x) pp[x + 1] += pp[x];
    int32_t* plus = (int32_t*)malloc((size_t)(pp[n] > 0 ? pp[n] : 1) * sizeof(int32_t));
#pragma omp parallel for schedule(dynamic, 4096)
    for (int32_t x = 0; x < n; ++x) {
        int64_t p = pp[x];
        for (int32_t j = rowptr[x]; j < rowptr[x + 1]; ++j)
            if (ORC_BEFORE(x, col[j])) plus[p++] = col[j];
    }
#undef ORC_BEFORE
    for (int32_t x = 0; x < n; ++x) counts[x] = 0;
    int64_t total = 0;
    const size_t words = ((size_t)n + 63) / 64;
#pragma omp parallel reduction(+ : total)
    {
        uint64_t* mark = (uint64_t*)calloc(words, sizeof(uint64_t));
        int64_t* t = (int64_t*)calloc((size_t)n, sizeof(int64_t));
#pragma omp for schedule(dynamic, 64)
        for (int32_t x = 0; x < n; ++x) {
            for (int64_t j = pp[x]; j < pp[x + 1]; ++j) mark[plus[j] >> 6] |= 1ull << (plus[j] & 63);
            int64_t tx = 0;
            for (int64_t j = pp[x]; j < pp[x + 1]; ++j) {
                const int32_t v = plus[j];
                int64_t tv = 0;
                for (int64_t k = pp[v]; k < pp[v + 1]; ++k) {
                    const int32_t w = plus[k];
                    if ((mark[w >> 6] >> (w & 63)) & 1u) {
                        ++tv;
                        ++t[w];
                    }
                }
                t[v] += tv;
                tx += tv;
            }
            for (int64_t j = pp[x]; j < pp[x + 1]; ++j) mark[plus[j] >> 6] = 0;
            t[x] += tx;
            total += tx;
        }
#pragma omp critical
        for (int32_t x = 0; x < n; ++x) counts[x] += t[x];
        free(mark);
        free(t);
    }
    for (int32_t x = 0; x < n; ++x) counts[x] *= 6;
    free(plus);
    free(pp);
    return total;
}

/*
 * CPU oracle for D-core ((k,l)-core) decomposition -- TEST INFRASTRUCTURE.
 *
 * This file is the checker, not the product.  Only the test suite, the smoke
 * check and the CPU-baseline leg of the benchmark load it; the engine never
 * calls it and has no CPU fallback through it.
 *
 * The reference (llysdal/d-core-cuda) has no CPU D-core code: src/graph_cpu.cpp
 * is only a text loader (src/graph_cpu.cpp:38-102).  Its decomposition lives
 * in CUDA kernels, so this file restates that algorithm on the CPU:
 *
 *   or_peel_levels  literal, sequential restatement of one reference pass:
 *                   the level loop of KList/KListInplace (main.cu:144-195)
 *                   around the `scan` seed (main.cu:27-62) and the `process`
 *                   cascade (main.cu:72-141).  O(V * levels + E) per pass,
 *                   used on small graphs to pin the fast variant below.
 *   or_bz_row       the same pass as a bucket-queue peel (Batagelj &
 *                   Zaversnik 2003, adapted to the in-degree >= k constraint)
 *                   restricted to C_k = {v : kmax[v] >= k}.  O(V + E).
 *   or_dcore        dcore(Graph&) (main.cu:197-262): kmax via the in/out
 *                   swapped k=0 pass (common.h:114-120, main.cu:218-220),
 *                   then rows k = 0..kmax (main.cu:238-244).
 *
 * Semantics pinned by the reference's golden decomposition of
 * dataset/digraph (dataset/digraph.decomp).  Maintenance has no separate
 * oracle: the reference's own tests compare maintained results against a full
 * recomputation on the updated graph (main.cu:2116-2143, checkDCore
 * main.cu:276-293), which is what the tests here do with or_dcore.
 *
 * Degrees are int32 (`degree` in src/common.h:59), vertex ids uint32.
 * Multi-edges are kept and counted, as the reference's text loader keeps
 * duplicate edges (src/graph.cpp:160-168).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_OK 0
#define OR_ERR_INVALID (-1)
#define OR_ERR_NOMEM (-3)
#define OR_ERR_CAPACITY (-5)

typedef struct {
    uint32_t V;
    uint64_t E;
    uint64_t* out_off; /* V+1 */
    uint32_t* out_nbr; /* E   */
    uint64_t* in_off;  /* V+1 */
    uint32_t* in_nbr;  /* E   */
} or_graph;

static void or_graph_free(or_graph* g) {
    free(g->out_off); free(g->out_nbr); free(g->in_off); free(g->in_nbr);
    memset(g, 0, sizeof(*g));
}

/* CSR (out) + CSC (in) with the input order kept inside each list. */
static int or_graph_build(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, or_graph* g) {
    memset(g, 0, sizeof(*g));
    g->V = V; g->E = E;
    g->out_off = (uint64_t*)calloc((size_t)V + 1, sizeof(uint64_t));
    g->in_off = (uint64_t*)calloc((size_t)V + 1, sizeof(uint64_t));
    g->out_nbr = (uint32_t*)malloc((E ? E : 1) * sizeof(uint32_t));
    g->in_nbr = (uint32_t*)malloc((E ? E : 1) * sizeof(uint32_t));
    if (!g->out_off || !g->in_off || !g->out_nbr || !g->in_nbr) { or_graph_free(g); return OR_ERR_NOMEM; }
    for (uint64_t e = 0; e < E; ++e) {
        if (src[e] >= V || dst[e] >= V) { or_graph_free(g); return OR_ERR_INVALID; }
        g->out_off[src[e] + 1]++;
        g->in_off[dst[e] + 1]++;
    }
    for (uint32_t v = 0; v < V; ++v) { g->out_off[v + 1] += g->out_off[v]; g->in_off[v + 1] += g->in_off[v]; }
    uint64_t* oc = (uint64_t*)malloc(((size_t)V + 1) * sizeof(uint64_t));
    uint64_t* ic = (uint64_t*)malloc(((size_t)V + 1) * sizeof(uint64_t));
    if (!oc || !ic) { free(oc); free(ic); or_graph_free(g); return OR_ERR_NOMEM; }
    memcpy(oc, g->out_off, ((size_t)V + 1) * sizeof(uint64_t));
    memcpy(ic, g->in_off, ((size_t)V + 1) * sizeof(uint64_t));
    for (uint64_t e = 0; e < E; ++e) {
        g->out_nbr[oc[src[e]]++] = dst[e];
        g->in_nbr[ic[dst[e]]++] = src[e];
    }
    free(oc); free(ic);
    return OR_OK;
}

/*
 * Literal restatement of one reference pass (KListInplace, main.cu:171-195).
 * swap != 0 exchanges the roles of in and out lists first (swapInOut,
 * common.h:114-120), which turns the pass into the kmax pass.
 * Level loop: while (count < V) { scan; process; level++ }  (main.cu:181-189)
 *   scan    (main.cu:37-56): unvisited v with out_deg == level is peeled;
 *           else unvisited v with in_deg < k is peeled and out_deg := level.
 *   process (main.cu:100-135): for each peeled v, every out-neighbour u gets
 *           in_deg[u]--; if the old value was k, u is peeled at this level.
 *           Every in-neighbour w gets out_deg[w]--; if the old value was
 *           level+1, w is peeled at this level.
 * Returns level-1 (the last level that ran), like KListInplace; -1 for V=0.
 */
int32_t or_peel_levels(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                       int swap, int32_t k, int32_t* core) {
    or_graph g;
    if (or_graph_build(V, E, swap ? dst : src, swap ? src : dst, &g) != OR_OK) return -2;
    int32_t* outdeg = (int32_t*)malloc(((size_t)V + 1) * sizeof(int32_t));
    int32_t* indeg = (int32_t*)malloc(((size_t)V + 1) * sizeof(int32_t));
    uint8_t* visited = (uint8_t*)calloc((size_t)V + 1, 1);
    uint32_t* queue = (uint32_t*)malloc(((size_t)V + 1) * sizeof(uint32_t));
    for (uint32_t v = 0; v < V; ++v) {
        outdeg[v] = (int32_t)(g.out_off[v + 1] - g.out_off[v]);
        indeg[v] = (int32_t)(g.in_off[v + 1] - g.in_off[v]);
        core[v] = -1;
    }
    uint64_t count = 0;
    int32_t level = 0;
    while (count < V) {
        size_t head = 0, tail = 0;
        for (uint32_t v = 0; v < V; ++v) {
            if (visited[v]) continue;
            if (outdeg[v] == level) {
                visited[v] = 1; queue[tail++] = v; core[v] = level;
            } else if (indeg[v] < k) {
                visited[v] = 1; queue[tail++] = v; outdeg[v] = level; core[v] = level;
            }
        }
        while (head < tail) {
            uint32_t v = queue[head++];
            for (uint64_t o = g.out_off[v]; o < g.out_off[v + 1]; ++o) {
                uint32_t u = g.out_nbr[o];
                int32_t old = indeg[u]--;
                if (old == k && !visited[u]) { visited[u] = 1; queue[tail++] = u; core[u] = level; }
            }
            for (uint64_t o = g.in_off[v]; o < g.in_off[v + 1]; ++o) {
                uint32_t w = g.in_nbr[o];
                int32_t old = outdeg[w]--;
                if (old == level + 1 && !visited[w]) { visited[w] = 1; queue[tail++] = w; core[w] = level; }
            }
        }
        count += tail;
        level++;
    }
    free(outdeg); free(indeg); free(visited); free(queue);
    or_graph_free(&g);
    return level - 1;
}

/* ---------------------------------------------------------------------- */
/* Bucket-queue pass                                                       */
/* ---------------------------------------------------------------------- */

enum { ST_DEAD = 0, ST_ALIVE = 1, ST_FORCED = 2, ST_DONE = 3 };

typedef struct {
    int32_t* key;   /* peeling degree (out-degree inside C_k) */
    int32_t* cdeg;  /* constraint degree (in-degree inside C_k) */
    uint32_t* vert;
    uint32_t* pos;
    uint64_t* bin;
    uint32_t* stack;
    uint8_t* st;
    size_t bin_cap;
} or_scratch;

static int scratch_init(or_scratch* s, uint32_t V, uint64_t maxdeg) {
    memset(s, 0, sizeof(*s));
    size_t n = (size_t)V + 1;
    s->key = (int32_t*)malloc(n * sizeof(int32_t));
    s->cdeg = (int32_t*)malloc(n * sizeof(int32_t));
    s->vert = (uint32_t*)malloc(n * sizeof(uint32_t));
    s->pos = (uint32_t*)malloc(n * sizeof(uint32_t));
    s->stack = (uint32_t*)malloc(n * sizeof(uint32_t));
    s->st = (uint8_t*)malloc(n);
    s->bin_cap = (size_t)maxdeg + 2;
    s->bin = (uint64_t*)malloc(s->bin_cap * sizeof(uint64_t));
    if (!s->key || !s->cdeg || !s->vert || !s->pos || !s->stack || !s->st || !s->bin) return OR_ERR_NOMEM;
    return OR_OK;
}
static void scratch_free(or_scratch* s) {
    free(s->key); free(s->cdeg); free(s->vert); free(s->pos); free(s->stack); free(s->st); free(s->bin);
    memset(s, 0, sizeof(*s));
}

/*
 * One pass over the set {v : member[v] >= k} (all vertices when member is
 * NULL).  a_off/a_nbr is the list whose length is peeled level by level (the
 * out-list for rows, the in-list for the kmax pass); b_off/b_nbr is the
 * opposite list.  Removing x lowers the peeling degree of every b-neighbour of
 * x and the constraint degree of every a-neighbour; a vertex whose constraint
 * degree falls below k leaves at the current level (the in_deg test of
 * main.cu:47,115).  Writes out[v] for every v (0 outside the set) and returns
 * the largest value written.
 */
static int32_t or_bz_pass(uint32_t V, const uint64_t* a_off, const uint32_t* a_nbr,
                          const uint64_t* b_off, const uint32_t* b_nbr,
                          const int32_t* member, int32_t k, int32_t* out, or_scratch* s) {
    int32_t maxkey = 0;
    uint32_t n = 0;
    for (uint32_t v = 0; v < V; ++v) {
        if (member && member[v] < k) { s->st[v] = ST_DEAD; out[v] = 0; continue; }
        s->st[v] = ST_ALIVE;
        n++;
    }
    for (uint32_t v = 0; v < V; ++v) {
        if (s->st[v] != ST_ALIVE) continue;
        int32_t kd = 0, cd = 0;
        for (uint64_t o = a_off[v]; o < a_off[v + 1]; ++o) kd += (s->st[a_nbr[o]] != ST_DEAD);
        for (uint64_t o = b_off[v]; o < b_off[v + 1]; ++o) cd += (s->st[b_nbr[o]] != ST_DEAD);
        s->key[v] = kd;
        s->cdeg[v] = cd;
        if (kd > maxkey) maxkey = kd;
    }
    if (n == 0) return 0;
    /* counting sort by key */
    memset(s->bin, 0, ((size_t)maxkey + 2) * sizeof(uint64_t));
    for (uint32_t v = 0; v < V; ++v) if (s->st[v] == ST_ALIVE) s->bin[s->key[v] + 1]++;
    for (int32_t d = 0; d <= maxkey; ++d) s->bin[d + 1] += s->bin[d];
    for (uint32_t v = 0; v < V; ++v) {
        if (s->st[v] != ST_ALIVE) continue;
        uint64_t p = s->bin[s->key[v]]++;
        s->vert[p] = v; s->pos[v] = (uint32_t)p;
    }
    for (int32_t d = maxkey; d > 0; --d) s->bin[d] = s->bin[d - 1];
    s->bin[0] = 0;

    int32_t level = 0, best = 0;
    size_t sp = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t v = s->vert[i];
        if (s->st[v] != ST_ALIVE) continue;
        if (s->key[v] > level) level = s->key[v];
        s->stack[sp++] = v;
        s->st[v] = ST_FORCED;
        while (sp) {
            uint32_t x = s->stack[--sp];
            s->st[x] = ST_DONE;
            out[x] = level;
            if (level > best) best = level;
            /* x's a-neighbours lose one unit of constraint degree */
            for (uint64_t o = a_off[x]; o < a_off[x + 1]; ++o) {
                uint32_t u = a_nbr[o];
                if (s->st[u] != ST_ALIVE) continue;
                if (--s->cdeg[u] < k) { s->st[u] = ST_FORCED; s->stack[sp++] = u; }
            }
            /* x's b-neighbours lose one unit of peeling degree */
            for (uint64_t o = b_off[x]; o < b_off[x + 1]; ++o) {
                uint32_t w = b_nbr[o];
                if (s->st[w] != ST_ALIVE) continue;
                int32_t d = s->key[w];
                if (d > level) {
                    uint64_t pw = s->pos[w], ps = s->bin[d];
                    uint32_t u = s->vert[ps];
                    if (u != w) { s->vert[pw] = u; s->pos[u] = (uint32_t)pw; s->vert[ps] = w; s->pos[w] = (uint32_t)ps; }
                    s->bin[d]++;
                    s->key[w] = d - 1;
                }
            }
        }
    }
    return best;
}

static uint64_t max_list(uint32_t V, const uint64_t* off) {
    uint64_t m = 0;
    for (uint32_t v = 0; v < V; ++v) if (off[v + 1] - off[v] > m) m = off[v + 1] - off[v];
    return m;
}

/* In-degree core numbers (the swapped k = 0 pass of dcore, main.cu:218-220). */
int32_t or_kmax(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, int32_t* kmaxes) {
    or_graph g;
    if (or_graph_build(V, E, src, dst, &g) != OR_OK) return -2;
    or_scratch s;
    if (scratch_init(&s, V, max_list(V, g.in_off)) != OR_OK) { scratch_free(&s); or_graph_free(&g); return -2; }
    int32_t km = or_bz_pass(V, g.in_off, g.in_nbr, g.out_off, g.out_nbr, NULL, 0, kmaxes, &s);
    scratch_free(&s);
    or_graph_free(&g);
    return km;
}

/* One row of the decomposition: out[v] = lmax_k(v), 0 outside C_k. */
int32_t or_bz_row(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst,
                  const int32_t* kmaxes, int32_t k, int32_t* out) {
    or_graph g;
    if (or_graph_build(V, E, src, dst, &g) != OR_OK) return -2;
    or_scratch s;
    if (scratch_init(&s, V, max_list(V, g.out_off)) != OR_OK) { scratch_free(&s); or_graph_free(&g); return -2; }
    int32_t l = or_bz_pass(V, g.out_off, g.out_nbr, g.in_off, g.in_nbr, kmaxes, k, out, &s);
    scratch_free(&s);
    or_graph_free(&g);
    return l;
}

/*
 * Full decomposition (dcore, main.cu:197-262).
 *   kmaxes_out[V]                 in-degree core numbers
 *   lmaxes_out[(kmax+1) * V]      row k = lmax_k, row-major
 * If lmaxes_out is NULL or rows_cap < kmax+1 the call only reports *kmax and
 * returns OR_ERR_CAPACITY (size query).  Rows run in parallel over `threads`
 * OpenMP threads (<= 0: all), largest rows first.
 */
int or_dcore_timed(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, int threads,
                   int32_t* kmaxes_out, int32_t* lmaxes_out, uint64_t rows_cap,
                   int32_t* kmax_out, int32_t* lmax_out, double* seconds);

int or_dcore(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, int threads,
             int32_t* kmaxes_out, int32_t* lmaxes_out, uint64_t rows_cap,
             int32_t* kmax_out, int32_t* lmax_out) {
    return or_dcore_timed(V, E, src, dst, threads, kmaxes_out, lmaxes_out, rows_cap, kmax_out, lmax_out, NULL);
}

/*
 * or_dcore that also reports, in *seconds (may be NULL), the wall time of the
 * decomposition itself: from the built CSR/CSC (the reference's dcore() gets
 * its Graph already in that form, main.cu:197) to the last row.
 */
int or_dcore_timed(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, int threads,
                   int32_t* kmaxes_out, int32_t* lmaxes_out, uint64_t rows_cap,
                   int32_t* kmax_out, int32_t* lmax_out, double* seconds) {
    or_graph g;
    int rc = or_graph_build(V, E, src, dst, &g);
    if (rc != OR_OK) return rc;
#ifdef _OPENMP
    const double t_start = omp_get_wtime();
#endif
    if (seconds) *seconds = 0.0;
    or_scratch s0;
    uint64_t md = max_list(V, g.in_off), mo = max_list(V, g.out_off);
    if (scratch_init(&s0, V, md > mo ? md : mo) != OR_OK) { scratch_free(&s0); or_graph_free(&g); return OR_ERR_NOMEM; }
    int32_t km = V ? or_bz_pass(V, g.in_off, g.in_nbr, g.out_off, g.out_nbr, NULL, 0, kmaxes_out, &s0) : 0;
    scratch_free(&s0);
    *kmax_out = km;
    if (!lmaxes_out || rows_cap < (uint64_t)km + 1) { or_graph_free(&g); return OR_ERR_CAPACITY; }
    int32_t lm = 0;
    int nt = threads;
#ifdef _OPENMP
    if (nt <= 0) nt = omp_get_max_threads();
#else
    nt = 1;
#endif
    if (nt > km + 1) nt = km + 1;
    int failed = 0;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt) reduction(max : lm) reduction(| : failed)
#endif
    {
        or_scratch s;
        if (scratch_init(&s, V, mo) != OR_OK) failed = 1;
        else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int32_t k = 0; k <= km; ++k) {
                int32_t l = or_bz_pass(V, g.out_off, g.out_nbr, g.in_off, g.in_nbr, kmaxes_out, k,
                                       lmaxes_out + (uint64_t)k * V, &s);
                if (l > lm) lm = l;
            }
        }
        scratch_free(&s);
    }
#ifdef _OPENMP
    if (seconds) *seconds = omp_get_wtime() - t_start;
#endif
    or_graph_free(&g);
    if (failed) return OR_ERR_NOMEM;
    *lmax_out = lm;
    return OR_OK;
}

/*
 * Edge-batch partition of getKmaxEdgeBatches with KEDGE_BATCHING
 * (main.cu:1441-1488).  Each edge's root is the endpoint with the larger kmax
 * (ties go to the target, main.cu:1450-1452); edges are bucketed by the
 * root's kmax in ascending order, and each bucket is split greedily, in input
 * order, into sub-batches with pairwise distinct roots.
 *   batch_of[e]   index of the sub-batch edge e lands in
 * Returns the number of sub-batches.
 */
int64_t or_kedge_batches(uint32_t V, const int32_t* kmaxes, uint64_t B,
                         const uint32_t* from, const uint32_t* to, int64_t* batch_of) {
    if (B == 0) return 0;
    int32_t maxk = 0;
    uint32_t* root = (uint32_t*)malloc(B * sizeof(uint32_t));
    int32_t* rk = (int32_t*)malloc(B * sizeof(int32_t));
    for (uint64_t e = 0; e < B; ++e) {
        uint32_t r = to[e];
        if (kmaxes[from[e]] > kmaxes[to[e]]) r = from[e];
        root[e] = r;
        rk[e] = kmaxes[r];
        if (rk[e] > maxk) maxk = rk[e];
    }
    uint8_t* used = (uint8_t*)calloc(V ? V : 1, 1);
    uint8_t* taken = (uint8_t*)calloc(B, 1);
    uint64_t* members = (uint64_t*)malloc(B * sizeof(uint64_t));
    int64_t nb = 0;
    /* bucket lists in input order */
    uint64_t* cnt = (uint64_t*)calloc((size_t)maxk + 2, sizeof(uint64_t));
    for (uint64_t e = 0; e < B; ++e) cnt[rk[e] + 1]++;
    for (int32_t d = 0; d <= maxk; ++d) cnt[d + 1] += cnt[d];
    uint64_t* order = (uint64_t*)malloc(B * sizeof(uint64_t));
    uint64_t* fill = (uint64_t*)malloc(((size_t)maxk + 2) * sizeof(uint64_t));
    memcpy(fill, cnt, ((size_t)maxk + 2) * sizeof(uint64_t));
    for (uint64_t e = 0; e < B; ++e) order[fill[rk[e]]++] = e;
    for (int32_t d = 0; d <= maxk; ++d) {
        uint64_t lo = cnt[d], hi = cnt[d + 1];
        uint64_t left = hi - lo;
        while (left) {
            uint64_t m = 0;
            for (uint64_t i = lo; i < hi; ++i) {
                uint64_t e = order[i];
                if (taken[e]) continue;
                if (m == 0 || !used[root[e]]) {
                    used[root[e]] = 1;
                    taken[e] = 1;
                    batch_of[e] = nb;
                    members[m++] = e;
                }
            }
            for (uint64_t i = 0; i < m; ++i) used[root[members[i]]] = 0;
            left -= m;
            nb++;
        }
    }
    free(root); free(rk); free(used); free(taken); free(members); free(cnt); free(order); free(fill);
    return nb;
}

/*
 * CPU-baseline sample: rows k = 0, stride, 2*stride, ... <= kmax of the
 * decomposition above, in parallel over `threads` threads (<= 0: all), each
 * into a per-thread scratch row.  Returns the number of rows computed (or a
 * negative error); *row_seconds receives the summed per-row wall time.  Used to time the CPU path on a bounded share of a large
 * decomposition; the full time is extrapolated by the caller.
 */
int64_t or_rows_sample(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, int threads,
                       const int32_t* kmaxes, int32_t kmax, int32_t stride, double* row_seconds) {
    or_graph g;
    if (or_graph_build(V, E, src, dst, &g) != OR_OK) return -2;
    uint64_t mo = max_list(V, g.out_off);
    int nt = threads;
#ifdef _OPENMP
    if (nt <= 0) nt = omp_get_max_threads();
#else
    nt = 1;
#endif
    if (stride < 1) stride = 1;
    int64_t nrows = (int64_t)kmax / stride + 1;
    if (nt > nrows) nt = (int)nrows;
    int failed = 0;
    double secs = 0.0;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt) reduction(| : failed) reduction(+ : secs)
#endif
    {
        or_scratch s;
        int32_t* out = (int32_t*)malloc(((size_t)V + 1) * sizeof(int32_t));
        if (scratch_init(&s, V, mo) != OR_OK || !out) failed = 1;
        else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int64_t r = 0; r < nrows; ++r) {
                int32_t k = (int32_t)(r * stride);
#ifdef _OPENMP
                double t0 = omp_get_wtime();
#endif
                or_bz_pass(V, g.out_off, g.out_nbr, g.in_off, g.in_nbr, kmaxes, k, out, &s);
#ifdef _OPENMP
                secs += omp_get_wtime() - t0;
#endif
            }
        }
        free(out);
        scratch_free(&s);
    }
    or_graph_free(&g);
    if (row_seconds) *row_seconds = secs;
    return failed ? -3 : nrows;
}

/* Number of threads the oracle's parallel regions use by default. */
int or_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/*
 * A built graph kept between calls, for checking a large decomposition a few
 * rows at a time (dense rows of a scale-24 graph do not fit in host memory at
 * once): or_graph_new builds the CSR/CSC once, or_graph_rows computes rows
 * k0 .. k1-1 (dcore's per-row pass, main.cu:236-243, rows in parallel) into
 * out[(k1 - k0) * V] from the given kmax values, or_graph_kmax the kmax
 * pass.  The rows are those of or_dcore.
 */
void* or_graph_new(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst) {
    or_graph* g = (or_graph*)malloc(sizeof(or_graph));
    if (!g) return NULL;
    if (or_graph_build(V, E, src, dst, g) != OR_OK) { free(g); return NULL; }
    return g;
}

void or_graph_delete(void* gp) {
    if (!gp) return;
    or_graph_free((or_graph*)gp);
    free(gp);
}

int32_t or_graph_kmax(void* gp, int32_t* kmaxes) {
    or_graph* g = (or_graph*)gp;
    or_scratch s;
    if (scratch_init(&s, g->V, max_list(g->V, g->in_off)) != OR_OK) { scratch_free(&s); return -2; }
    int32_t km = g->V ? or_bz_pass(g->V, g->in_off, g->in_nbr, g->out_off, g->out_nbr, NULL, 0, kmaxes, &s) : 0;
    scratch_free(&s);
    return km;
}

int or_graph_rows(void* gp, int threads, const int32_t* kmaxes, int32_t k0, int32_t k1, int32_t* out) {
    or_graph* g = (or_graph*)gp;
    const uint32_t V = g->V;
    uint64_t mo = max_list(V, g->out_off);
    int nt = threads;
#ifdef _OPENMP
    if (nt <= 0) nt = omp_get_max_threads();
#else
    nt = 1;
#endif
    if (k1 <= k0) return OR_OK;
    if (nt > k1 - k0) nt = k1 - k0;
    int failed = 0;
#ifdef _OPENMP
#pragma omp parallel num_threads(nt) reduction(| : failed)
#endif
    {
        or_scratch s;
        if (scratch_init(&s, V, mo) != OR_OK) failed = 1;
        else {
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
            for (int32_t k = k0; k < k1; ++k)
                or_bz_pass(V, g->out_off, g->out_nbr, g->in_off, g->in_nbr, kmaxes, k, out + (uint64_t)(k - k0) * V, &s);
        }
        scratch_free(&s);
    }
    return failed ? OR_ERR_NOMEM : OR_OK;
}

/*
 * vann_oracle.c -- CPU restatement of the reference's Vamana hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker, see vann_oracle.h).  Pinned
 * against the reference's golden graph vamana/vout/vamana.out, which this code
 * rebuilds from data/sift10k/sift10k_randomgraph.bin (tests/test_oracle_golden.py).
 */
#include "vann_oracle.h"

#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- bloom filter
 * vamana/include/bloom_filter.cuh:11-30: FNV-style byte folding in 64-bit
 * arithmetic, reduced modulo 39,988 slots.  The seeds and primes are the
 * reference's; they have to be identical for the filter's false positives, and
 * so the search trajectories, to be identical. */
uint32_t vo_bf_h1(uint32_t x) {
    uint64_t h = 0xcbf29ce4ull;
    for (int s = 0; s < 32; s += 8) h = (h ^ ((x >> s) & 0xffu)) * 0x01000193ull;
    return (uint32_t)(h % VO_BF_ENTRIES);
}

uint32_t vo_bf_h2(uint32_t x) {
    uint64_t h = 0x84222325ull;
    for (int s = 0; s < 32; s += 8) h = (h ^ ((x >> s) & 0xffu)) * 0x1B3ull;
    return (uint32_t)(h % VO_BF_ENTRIES);
}

/* Squared L2 in FP32 (kernels.cuh:14-54, utils.cuh:150-158).  Sequential over
 * the dimension.  For integer-valued vectors with sums below 2^24 every order
 * gives the same bits. */
float vo_l2sq(const float* a, const float* b, int dim) {
    float s = 0.0f;
    for (int i = 0; i < dim; ++i) {
        float d = a[i] - b[i];
        s       = fmaf(d, d, s);
    }
    return s;
}

static inline int tomb_get(const uint32_t* t, uint32_t id) {
    return t && ((t[id >> 5] >> (id & 31)) & 1u);
}

/* ---------------------------------------------------------------- sorting
 * (dist, id) ascending for one expansion's new neighbours; (dist, position)
 * ascending (= stable by distance) for candidate lists (kernels.cuh:82-139). */
typedef struct {
    float    d;
    uint32_t id;
    uint32_t pos;
} vo_item;

static int cmp_dist_id(const void* a, const void* b) {
    const vo_item* x = (const vo_item*)a;
    const vo_item* y = (const vo_item*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->id > y->id) - (x->id < y->id);
}

static int cmp_dist_pos(const void* a, const void* b) {
    const vo_item* x = (const vo_item*)a;
    const vo_item* y = (const vo_item*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->pos > y->pos) - (x->pos < y->pos);
}

/* ---------------------------------------------------------------- GreedySearch */
int vo_search_one(const vo_graph* g, const float* q, int L, uint32_t entry, uint32_t skip_id,
                  int bloom_mode, int max_visited, int max_hops, uint32_t* wl_ids, float* wl_d,
                  int* wl_n, uint32_t* vis_ids, float* vis_d, int* vis_n, int* hops_out,
                  int64_t* evals_out, int64_t* adjw_out) {
    const int     D   = g->dim;
    const int     R   = g->R;
    unsigned char* bf = (unsigned char*)calloc(VO_BF_ENTRIES, 1);
    unsigned char* wl_v = (unsigned char*)calloc((size_t)L, 1);
    vo_item*       nb   = (vo_item*)malloc(sizeof(vo_item) * (size_t)(R > 0 ? R : 1));
    uint32_t*      tmp_i = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)L);
    float*         tmp_d = (float*)malloc(sizeof(float) * (size_t)L);
    unsigned char* tmp_v = (unsigned char*)malloc((size_t)L);
    int*           pass = (int*)malloc(sizeof(int) * (size_t)(R > 0 ? R : 1));
    int            status = VO_OK;

    /* initializeWorklist (search.cuh:30-58): entry is in the worklist, marked
     * visited, but NOT in the bloom filter. */
    int     n     = 1;
    int64_t evals = 1;
    wl_ids[0]     = entry;
    wl_d[0]       = vo_l2sq(q, g->vecs + (size_t)entry * D, D);
    wl_v[0]       = 1;
    uint32_t parent   = entry;
    float    parent_d = wl_d[0];
    int      hops     = 0;
    int      nv       = 0;
    int64_t  adjw     = 0;

    for (;;) {
        if (hops >= max_hops) {
            status = VO_ERR_HOP_LIMIT;
            break;
        }
        ++hops;
        /* filterNeighbors (search.cuh:71-138): record the parent, then filter its
         * adjacency through the delete list, the batch-index skip and the bloom
         * filter. */
        if (nv < max_visited) {
            if (vis_ids) vis_ids[nv] = parent;
            if (vis_d) vis_d[nv] = parent_d;
            ++nv;
        }
        const uint32_t  deg = g->deg[parent] < (uint32_t)R ? g->deg[parent] : (uint32_t)R;
        const uint32_t* row = g->adj + (size_t)parent * R;
        adjw += deg;
        int             cnt = 0;
        const uint32_t  chunk = bloom_mode == VO_BLOOM_SEQUENTIAL ? 1u
                                : bloom_mode == VO_BLOOM_SNAPSHOT ? (deg ? deg : 1u)
                                                                  : 32u;
        for (uint32_t c0 = 0; c0 < deg; c0 += chunk) {
            uint32_t c1 = c0 + chunk < deg ? c0 + chunk : deg;
            for (uint32_t j = c0; j < c1; ++j) {
                uint32_t id = row[j];
                int      ok = !tomb_get(g->tomb, id) && id != skip_id;
                if (ok) {
                    uint32_t a = vo_bf_h1(id), b = vo_bf_h2(id);
                    ok = !(bf[a] && bf[b]);
                }
                pass[j - c0] = ok;
            }
            for (uint32_t j = c0; j < c1; ++j) {
                if (!pass[j - c0]) continue;
                uint32_t id = row[j];
                bf[vo_bf_h1(id)] = 1;
                bf[vo_bf_h2(id)] = 1;
                nb[cnt].id       = id;
                nb[cnt].d        = vo_l2sq(q, g->vecs + (size_t)id * D, D);
                ++cnt;
            }
        }
        evals += cnt;
        qsort(nb, (size_t)cnt, sizeof(vo_item), cmp_dist_id);

        /* mergeIntoWorklist (search.cuh:140-223): stable merge, existing entries
         * before new ones on equal distance, truncate to L. */
        int i = 0, j = 0, m = 0;
        while (m < L && (i < n || j < cnt)) {
            if (j >= cnt || (i < n && wl_d[i] <= nb[j].d)) {
                tmp_i[m] = wl_ids[i];
                tmp_d[m] = wl_d[i];
                tmp_v[m] = wl_v[i];
                ++i;
            } else {
                tmp_i[m] = nb[j].id;
                tmp_d[m] = nb[j].d;
                tmp_v[m] = 0;
                ++j;
            }
            ++m;
        }
        n = m;
        memcpy(wl_ids, tmp_i, sizeof(uint32_t) * (size_t)n);
        memcpy(wl_d, tmp_d, sizeof(float) * (size_t)n);
        memcpy(wl_v, tmp_v, (size_t)n);

        /* next parent: first unvisited entry (search.cuh:205-221) */
        int next = -1;
        for (int t = 0; t < n; ++t)
            if (!wl_v[t]) {
                next = t;
                break;
            }
        if (next < 0) break;
        wl_v[next] = 1;
        parent     = wl_ids[next];
        parent_d   = wl_d[next];
    }
    *wl_n = n;
    if (vis_n) *vis_n = nv;
    if (hops_out) *hops_out = hops;
    if (evals_out) *evals_out = evals;
    if (adjw_out) *adjw_out = adjw;
    free(bf);
    free(wl_v);
    free(nb);
    free(tmp_i);
    free(tmp_d);
    free(tmp_v);
    free(pass);
    return status;
}

int vo_search_batch(const vo_graph* g, const float* q, int64_t nq, int L, int k, uint32_t entry,
                    int skip_mode, int bloom_mode, int max_hops, uint32_t* out_ids, float* out_d,
                    int32_t* hops, int64_t* evals, int64_t* adjw, int threads) {
    if (L < 1 || k < 1 || k > L || g->R > 64 * 1024) return VO_ERR_INVALID;
    int status = VO_OK;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads)
    {
        uint32_t* wi = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)L);
        float*    wd = (float*)malloc(sizeof(float) * (size_t)L);
#pragma omp for schedule(dynamic, 16)
        for (int64_t s = 0; s < nq; ++s) {
            int      wn = 0, h = 0;
            int64_t  e = 0, aw = 0;
            uint32_t skip = skip_mode == 1 ? (uint32_t)s : VO_NONE;
            int st = vo_search_one(g, q + (size_t)s * g->dim, L, entry, skip, bloom_mode, 0,
                                   max_hops, wi, wd, &wn, NULL, NULL, NULL, &h, &e, &aw);
            if (st != VO_OK) {
#pragma omp atomic write
                status = st;
            }
            for (int t = 0; t < k; ++t) {
                out_ids[(size_t)s * k + t] = t < wn ? wi[t] : VO_NONE;
                out_d[(size_t)s * k + t]   = t < wn ? wd[t] : INFINITY;
            }
            if (hops) hops[s] = h;
            if (evals) evals[s] = e;
            if (adjw) adjw[s] = aw;
        }
        free(wi);
        free(wd);
    }
    return status;
}

/* ---------------------------------------------------------------- RobustPrune
 * kernels.cuh:232-356 / :626-743.  Candidates are sorted by distance to the
 * node.  Repeat: p* = first INIT candidate, append it, mark it NEIGHBOR, and
 * mark PRUNED every INIT p with dist(p*,p) * alpha <= dist(node,p) (squared
 * FP32 distances, product rounded to FP32), until R neighbours or no INIT. */
int vo_robust_prune(const vo_graph* g, const float* node_vec, const uint32_t* cand,
                    const float* cand_d, int nc, float alpha, int R, uint32_t* out,
                    int64_t* evals) {
    (void)node_vec;
    enum { INIT = 0, PRUNED = 1, NEIGHBOR = 2 };
    unsigned char* st  = (unsigned char*)calloc((size_t)(nc > 0 ? nc : 1), 1);
    int            deg = 0;
    int            first = 0;
    int64_t        ev    = 0;
    const int      D     = g->dim;
    while (deg < R) {
        while (first < nc && st[first] != INIT) ++first;
        if (first >= nc) break;
        uint32_t ps = cand[first];
        out[deg++]  = ps;
        st[first]   = NEIGHBOR;
        const float* pv = g->vecs + (size_t)ps * D;
        for (int t = first + 1; t < nc; ++t) {
            if (st[t] != INIT) continue;
            float dd = vo_l2sq(g->vecs + (size_t)cand[t] * D, pv, D);
            ++ev;
            float lhs = dd * alpha;
            if (lhs <= cand_d[t]) st[t] = PRUNED;
        }
    }
    if (evals) *evals += ev;
    free(st);
    return deg;
}

/* merge two lists sorted by distance; entries of `a` go first on ties; cap. */
static int merge_cap(const vo_item* a, int na, const vo_item* b, int nb, int cap,
                     uint32_t* out_id, float* out_d) {
    int i = 0, j = 0, m = 0;
    while (m < cap && (i < na || j < nb)) {
        if (j >= nb || (i < na && a[i].d <= b[j].d)) {
            out_id[m] = a[i].id;
            out_d[m]  = a[i].d;
            ++i;
        } else {
            out_id[m] = b[j].id;
            out_d[m]  = b[j].d;
            ++j;
        }
        ++m;
    }
    return m;
}

/* the node's current out-neighbours with distances, stable-sorted
 * (getNeighbors + computeDists + sortByDistance, kernels.cuh:141-169,406-431) */
static int sorted_out(const vo_graph* g, int64_t node, const float* node_vec, vo_item* it) {
    uint32_t d = g->deg[node];
    for (uint32_t j = 0; j < d; ++j) {
        uint32_t id = g->adj[(size_t)node * g->R + j];
        it[j].id    = id;
        it[j].pos   = j;
        it[j].d     = vo_l2sq(node_vec, g->vecs + (size_t)id * g->dim, g->dim);
    }
    qsort(it, d, sizeof(vo_item), cmp_dist_pos);
    return (int)d;
}

/* ---------------------------------------------------------------- Vamana batch */
/* The batch's node ids: nodes[b] when given, else batch_start + b. */
static int batch_impl(vo_graph* g, const uint32_t* nodes, int64_t batch_start, int64_t batch_n, int L,
                      float alpha, uint32_t entry, int max_visited, int max_reverse, int skip_mode,
                      int bloom_mode, int threads);

int vo_vamana_batch(vo_graph* g, int64_t batch_start, int64_t batch_n, int L, float alpha,
                    uint32_t entry, int max_visited, int max_reverse, int skip_mode,
                    int bloom_mode, int threads) {
    if (batch_start < 0 || batch_n < 0 || batch_start + batch_n > g->n) return VO_ERR_INVALID;
    return batch_impl(g, NULL, batch_start, batch_n, L, alpha, entry, max_visited, max_reverse, skip_mode,
                      bloom_mode, threads);
}

/* A batch over any node ids (inserts into ids freed by a consolidation): the same steps,
 * with the reverse entries of each target in batch order. */
int vo_vamana_batch_ids(vo_graph* g, const uint32_t* nodes, int64_t batch_n, int L, float alpha,
                        uint32_t entry, int max_visited, int max_reverse, int skip_mode, int bloom_mode,
                        int threads) {
    if (batch_n < 0 || (batch_n > 0 && !nodes)) return VO_ERR_INVALID;
    for (int64_t b = 0; b < batch_n; ++b)
        if (nodes[b] >= (uint64_t)g->n) return VO_ERR_INVALID;
    return batch_impl(g, nodes, 0, batch_n, L, alpha, entry, max_visited, max_reverse, skip_mode, bloom_mode,
                      threads);
}

static int batch_impl(vo_graph* g, const uint32_t* nodes, int64_t batch_start, int64_t batch_n, int L,
                      float alpha, uint32_t entry, int max_visited, int max_reverse, int skip_mode,
                      int bloom_mode, int threads) {
    const int     R = g->R, D = g->dim;
    const int64_t N = g->n;
    if (L < 1 || R < 1 || max_visited < 1 || max_reverse < 1) return VO_ERR_INVALID;
    if (threads <= 0) threads = omp_get_max_threads();
    int status = VO_OK;

    /* 1. greedySearch for every batch node (vamana_impl.cuh:325-331) */
    uint32_t* vis   = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)batch_n * max_visited);
    float*    vis_d = (float*)malloc(sizeof(float) * (size_t)batch_n * max_visited);
    int*      vis_n = (int*)calloc((size_t)(batch_n ? batch_n : 1), sizeof(int));
#pragma omp parallel num_threads(threads)
    {
        uint32_t* wi = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)L);
        float*    wd = (float*)malloc(sizeof(float) * (size_t)L);
#pragma omp for schedule(dynamic, 16)
        for (int64_t b = 0; b < batch_n; ++b) {
            int64_t  node = (nodes ? (int64_t)nodes[b] : batch_start + b);
            uint32_t skip = skip_mode == 1   ? (uint32_t)b
                            : skip_mode == 2 ? (uint32_t)node
                                             : VO_NONE;
            int wn = 0;
            int st = vo_search_one(g, g->vecs + (size_t)node * D, L, entry, skip, bloom_mode,
                                   max_visited, 1 << 30, wi, wd, &wn, vis + (size_t)b * max_visited,
                                   vis_d + (size_t)b * max_visited, &vis_n[b], NULL, NULL, NULL);
            if (st != VO_OK) {
#pragma omp atomic write
                status = st;
            }
        }
        free(wi);
        free(wd);
    }

    /* 2. computeOutNeighbors (kernels.cuh:358-500): candidates = stable-sorted
     * expansion list merged with the stable-sorted current out-neighbours
     * (expansion entries first on ties), capped at max_visited; RobustPrune. */
    uint32_t* chosen   = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)batch_n * R);
    int*      chosen_n = (int*)calloc((size_t)(batch_n ? batch_n : 1), sizeof(int));
#pragma omp parallel num_threads(threads)
    {
        vo_item*  a  = (vo_item*)malloc(sizeof(vo_item) * (size_t)max_visited);
        vo_item*  o  = (vo_item*)malloc(sizeof(vo_item) * (size_t)R);
        uint32_t* ci = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)max_visited);
        float*    cd = (float*)malloc(sizeof(float) * (size_t)max_visited);
#pragma omp for schedule(dynamic, 16)
        for (int64_t b = 0; b < batch_n; ++b) {
            int64_t      node = (nodes ? (int64_t)nodes[b] : batch_start + b);
            const float* nv   = g->vecs + (size_t)node * D;
            int          na   = vis_n[b];
            for (int t = 0; t < na; ++t) {
                a[t].id  = vis[(size_t)b * max_visited + t];
                a[t].d   = vis_d[(size_t)b * max_visited + t];
                a[t].pos = (uint32_t)t;
            }
            qsort(a, (size_t)na, sizeof(vo_item), cmp_dist_pos);
            int no = sorted_out(g, node, nv, o);
            int nc = merge_cap(a, na, o, no, max_visited, ci, cd);
            chosen_n[b] =
                vo_robust_prune(g, nv, ci, cd, nc, alpha, R, chosen + (size_t)b * R, NULL);
        }
        free(a);
        free(o);
        free(ci);
        free(cd);
    }
    /* write the new adjacency (pruneOutNeighbors rewrites deg/nbr in place) and
     * append reverse edges p* <- node in ascending node order (capped). */
    uint32_t* rev   = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N * max_reverse);
    uint32_t* rev_n = (uint32_t*)calloc((size_t)(N ? N : 1), sizeof(uint32_t));
    for (int64_t b = 0; b < batch_n; ++b) {
        int64_t node  = (nodes ? (int64_t)nodes[b] : batch_start + b);
        g->deg[node] = (uint32_t)chosen_n[b];
        for (int t = 0; t < chosen_n[b]; ++t) {
            uint32_t p                     = chosen[(size_t)b * R + t];
            g->adj[(size_t)node * R + t]   = p;
            if (rev_n[p] < (uint32_t)max_reverse) rev[(size_t)p * max_reverse + rev_n[p]++] = (uint32_t)node;
        }
    }

    /* 3. computeReverseEdges (kernels.cuh:745-903): for every node, candidates =
     * stable-sorted reverse entries merged with the stable-sorted current
     * out-neighbours (reverse entries first on ties), capped at max_reverse;
     * RobustPrune again (always, whatever the count). */
    uint32_t* new_adj = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N * R);
    uint32_t* new_deg = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(N ? N : 1));
#pragma omp parallel num_threads(threads)
    {
        vo_item*  a  = (vo_item*)malloc(sizeof(vo_item) * (size_t)max_reverse);
        vo_item*  o  = (vo_item*)malloc(sizeof(vo_item) * (size_t)R);
        uint32_t* ci = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(max_reverse + R));
        float*    cd = (float*)malloc(sizeof(float) * (size_t)(max_reverse + R));
#pragma omp for schedule(dynamic, 64)
        for (int64_t v = 0; v < N; ++v) {
            const float* nv = g->vecs + (size_t)v * D;
            int          na = (int)rev_n[v];
            for (int t = 0; t < na; ++t) {
                uint32_t id = rev[(size_t)v * max_reverse + t];
                a[t].id     = id;
                a[t].pos    = (uint32_t)t;
                a[t].d      = vo_l2sq(nv, g->vecs + (size_t)id * D, D);
            }
            qsort(a, (size_t)na, sizeof(vo_item), cmp_dist_pos);
            int no = sorted_out(g, v, nv, o);
            int nc = merge_cap(a, na, o, no, max_reverse, ci, cd);
            new_deg[v] =
                (uint32_t)vo_robust_prune(g, nv, ci, cd, nc, alpha, R, new_adj + (size_t)v * R, NULL);
        }
        free(a);
        free(o);
        free(ci);
        free(cd);
    }
    for (int64_t v = 0; v < N; ++v) {
        g->deg[v] = new_deg[v];
        memcpy(g->adj + (size_t)v * R, new_adj + (size_t)v * R, sizeof(uint32_t) * new_deg[v]);
    }

    free(vis);
    free(vis_d);
    free(vis_n);
    free(chosen);
    free(chosen_n);
    free(rev);
    free(rev_n);
    free(new_adj);
    free(new_deg);
    return status;
}

/* ---------------------------------------------------------------- helpers */
static uint64_t splitmix64(uint64_t x) {
    /* SplitMix64 finaliser (Steele, Lea, Flood 2014) */
    uint64_t z = x + 0x9e3779b97f4a7c15ull;
    z          = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z          = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

void vo_random_graph(int64_t n, int R, uint64_t seed, uint32_t* deg, uint32_t* adj) {
    for (int64_t i = 0; i < n; ++i) {
        uint32_t d = n > 1 ? (uint32_t)R : 0u;
        deg[i]     = d;
        for (int j = 0; j < R; ++j) {
            uint64_t h = splitmix64(seed ^ ((uint64_t)i * (uint64_t)R + (uint64_t)j));
            adj[(size_t)i * R + j] =
                n > 1 ? (uint32_t)((i + 1 + (int64_t)(h % (uint64_t)(n - 1))) % n) : 0u;
        }
    }
}

int64_t vo_medoid(const float* vecs, int64_t n, int dim) {
    double* mean = (double*)calloc((size_t)dim, sizeof(double));
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) mean[d] += vecs[(size_t)i * dim + d];
    for (int d = 0; d < dim; ++d) mean[d] /= (double)n;
    int64_t best  = 0;
    double  bestd = INFINITY;
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (int d = 0; d < dim; ++d) {
            double t = vecs[(size_t)i * dim + d] - mean[d];
            s += t * t;
        }
        if (s < bestd) {
            bestd = s;
            best  = i;
        }
    }
    free(mean);
    return best;
}

void vo_bruteforce_knn(const float* base, int64_t n, const float* q, int64_t nq, int dim, int k,
                       uint32_t* out_ids, double* out_d, int threads) {
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 4)
    for (int64_t s = 0; s < nq; ++s) {
        uint32_t* bi = out_ids + (size_t)s * k;
        double*   bd = out_d + (size_t)s * k;
        for (int t = 0; t < k; ++t) {
            bi[t] = VO_NONE;
            bd[t] = INFINITY;
        }
        const float* qs = q + (size_t)s * dim;
        for (int64_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int d = 0; d < dim; ++d) {
                double t = (double)base[(size_t)i * dim + d] - (double)qs[d];
                acc += t * t;
            }
            if (acc < bd[k - 1] || (acc == bd[k - 1] && (uint32_t)i < bi[k - 1])) {
                int p = k - 1;
                while (p > 0 && (bd[p - 1] > acc || (bd[p - 1] == acc && bi[p - 1] > (uint32_t)i))) {
                    bd[p] = bd[p - 1];
                    bi[p] = bi[p - 1];
                    --p;
                }
                bd[p] = acc;
                bi[p] = (uint32_t)i;
            }
        }
    }
}

/* l2_distance_sq (vamana/include/utils.cuh:150-158): sequential over the
 * dimensions, `dist += diff * diff` -- which nvcc contracts to one fused
 * multiply-add per dimension, so fmaf here. */
static float vo_l2_seq(const float* a, const float* b, int dim) {
    float d = 0.0f;
    for (int i = 0; i < dim; ++i) {
        const float diff = a[i] - b[i];
        d                = fmaf(diff, diff, d);
    }
    return d;
}

void vo_merge_rerank(const float* vecs, int dim, const float* q, int64_t nq, const uint32_t* graph_ids,
                     int L, const float* insert_list, int64_t n_il, uint32_t* out_ids, float* out_d) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t qi = 0; qi < nq; ++qi) {
        const float* qv   = q + (size_t)qi * dim;
        float*       sd   = out_d + (size_t)qi * L;
        uint32_t*    sid  = out_ids + (size_t)qi * L;
        for (int k = 0; k < L; ++k) {
            sd[k]  = INFINITY;
            sid[k] = 0xFFFFFFFFu;
        }
        for (int64_t c = 0; c < L + n_il; ++c) {
            uint32_t     id;
            const float* row;
            if (c < L) {
                id = graph_ids[(size_t)qi * L + c];
                if (id == 0xFFFFFFFFu) continue;  /* a padded worklist slot */
                row = vecs + (size_t)id * dim;
            } else {
                id  = 0x80000000u | (uint32_t)(c - L);
                row = insert_list + (size_t)(c - L) * dim;
            }
            const float dist = vo_l2_seq(qv, row, dim);
            /* utils.cuh:226-241: first slot holding the largest value */
            float max_dist = -1.0f;
            int   max_k    = 0;
            for (int k = 0; k < L; ++k)
                if (sd[k] > max_dist) {
                    max_dist = sd[k];
                    max_k    = k;
                }
            if (dist < max_dist) {
                sd[max_k]  = dist;
                sid[max_k] = id;
            }
        }
        /* utils.cuh:265-283: bubble sort by distance (stable) */
        for (int i = 0; i < L - 1; ++i)
            for (int j = 0; j < L - i - 1; ++j)
                if (sd[j] > sd[j + 1]) {
                    float    td = sd[j];
                    uint32_t ti = sid[j];
                    sd[j]       = sd[j + 1];
                    sid[j]      = sid[j + 1];
                    sd[j + 1]   = td;
                    sid[j + 1]  = ti;
                }
    }
}

/* ---------------------------------------------------------------- delete consolidation
 * The reference never consolidates deletes: patchGraph (vamana_impl.cuh:182-265)
 * folds in inserts only, and deleted ids stay behind a delete list that every
 * search scans (search.cuh:121-123, delete_list.cuh:108-115).  FreshVamana's
 * consolidation is the published FreshDiskANN rule (Singh, Subramanya,
 * Krishnaswamy, Simhadri, "FreshDiskANN", 2021, Algorithm 4 "Delete"):
 *   for every live p with N_out(p) meeting the deleted set D:
 *     C = (N_out(p) \ D)  U  (U_{v in N_out(p) & D} N_out(v)),  minus D and p;
 *     N_out(p) = RobustPrune(p, C, alpha, R).
 * The paper leaves the order of C open.  This restatement fixes the order the
 * engine uses: p's list in its order, each deleted neighbour replaced where it
 * stands by its own out-neighbours in their order, repeats dropped (the first
 * occurrence stays), at most `cap` entries.  Distances to p are FP32 (vo_l2sq),
 * the list is sorted stably by distance and pruned with vo_robust_prune.  Every
 * candidate list is taken from the graph before any node is re-pruned.
 * Then the deleted ids that are not free yet get degree 0 and join the free
 * list in ascending order; a deleted entry point moves to the first live id in
 * the L = 32 worklist of a search for its vector, started at the lowest live
 * id, over the consolidated graph (the tombstones stay set).
 * g->tomb marks the deleted ids; is_free (n bytes, may be NULL) marks ids
 * freed by an earlier consolidation. */
int vo_consolidate(vo_graph* g, float alpha, int cap, const unsigned char* is_free, uint32_t entry,
                   uint32_t* new_entry, uint32_t* freed, int64_t* n_freed, int threads) {
    const int     R = g->R, D = g->dim;
    const int64_t N = g->n;
    if (!g->tomb || cap < 1 || R < 1) return VO_ERR_INVALID;
    if (threads <= 0) threads = omp_get_max_threads();
    uint32_t* new_adj = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(N ? N : 1) * R);
    int32_t*  new_deg = (int32_t*)malloc(sizeof(int32_t) * (size_t)(N ? N : 1));
#pragma omp parallel num_threads(threads)
    {
        uint32_t* seen = (uint32_t*)calloc((size_t)(N ? N : 1), sizeof(uint32_t));
        vo_item*  it   = (vo_item*)malloc(sizeof(vo_item) * (size_t)cap);
        uint32_t* ci   = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cap);
        float*    cd   = (float*)malloc(sizeof(float) * (size_t)cap);
#pragma omp for schedule(dynamic, 64)
        for (int64_t p = 0; p < N; ++p) {
            new_deg[p] = -1; /* unchanged */
            if (tomb_get(g->tomb, (uint32_t)p)) continue;
            const uint32_t  dp  = g->deg[p] < (uint32_t)R ? g->deg[p] : (uint32_t)R;
            const uint32_t* row = g->adj + (size_t)p * R;
            int             any = 0;
            for (uint32_t j = 0; j < dp && !any; ++j) any = tomb_get(g->tomb, row[j]);
            if (!any) continue;
            const uint32_t stamp = (uint32_t)p + 1u;
            int            nc    = 0;
#define VO_PUSH(u)                                                                  \
    do {                                                                            \
        uint32_t u_ = (u);                                                          \
        if (nc < cap && u_ != (uint32_t)p && !tomb_get(g->tomb, u_) && seen[u_] != stamp) { \
            seen[u_]   = stamp;                                                     \
            it[nc].id  = u_;                                                        \
            it[nc].pos = (uint32_t)nc;                                              \
            ++nc;                                                                   \
        }                                                                           \
    } while (0)
            for (uint32_t j = 0; j < dp && nc < cap; ++j) {
                const uint32_t v = row[j];
                if (!tomb_get(g->tomb, v)) {
                    VO_PUSH(v);
                } else {
                    const uint32_t  dv   = g->deg[v] < (uint32_t)R ? g->deg[v] : (uint32_t)R;
                    const uint32_t* rowv = g->adj + (size_t)v * R;
                    for (uint32_t t = 0; t < dv && nc < cap; ++t) VO_PUSH(rowv[t]);
                }
            }
#undef VO_PUSH
            const float* pv = g->vecs + (size_t)p * D;
            for (int t = 0; t < nc; ++t) it[t].d = vo_l2sq(pv, g->vecs + (size_t)it[t].id * D, D);
            qsort(it, (size_t)nc, sizeof(vo_item), cmp_dist_pos);
            for (int t = 0; t < nc; ++t) {
                ci[t] = it[t].id;
                cd[t] = it[t].d;
            }
            new_deg[p] = vo_robust_prune(g, pv, ci, cd, nc, alpha, R, new_adj + (size_t)p * R, NULL);
        }
        free(seen);
        free(it);
        free(ci);
        free(cd);
    }
    int64_t nf = 0;
    for (int64_t p = 0; p < N; ++p) {
        if (new_deg[p] >= 0) {
            g->deg[p] = (uint32_t)new_deg[p];
            memcpy(g->adj + (size_t)p * R, new_adj + (size_t)p * R, sizeof(uint32_t) * (size_t)new_deg[p]);
        }
        if (tomb_get(g->tomb, (uint32_t)p) && !(is_free && is_free[p])) {
            g->deg[p] = 0;
            if (freed) freed[nf] = (uint32_t)p;
            ++nf;
        }
    }
    free(new_adj);
    free(new_deg);
    if (n_freed) *n_freed = nf;
    uint32_t ne = entry;
    if (entry < (uint64_t)N && tomb_get(g->tomb, entry)) {
        uint32_t start = VO_NONE;
        for (int64_t i = 0; i < N && start == VO_NONE; ++i)
            if (!tomb_get(g->tomb, (uint32_t)i)) start = (uint32_t)i;
        if (start == VO_NONE) return VO_ERR_INVALID;
        uint32_t wi[32];
        float    wd[32];
        int      wn = 0;
        int st = vo_search_one(g, g->vecs + (size_t)entry * D, 32, start, VO_NONE, VO_BLOOM_SNAPSHOT, 0,
                               1 << 30, wi, wd, &wn, NULL, NULL, NULL, NULL, NULL, NULL);
        if (st != VO_OK) return st;
        ne = start;
        for (int t = 0; t < wn; ++t)
            if (!tomb_get(g->tomb, wi[t])) {
                ne = wi[t];
                break;
            }
    }
    if (new_entry) *new_entry = ne;
    return VO_OK;
}

/* ---------------------------------------------------------------- uint8 grid */
/* The product's uint8 copy of float rows (cs5013-project_b200/csrc/graph_ops.cu
 * launch_u8_grid, convert_kernel; queries: csrc/rerank.cu grid_queries_kernel),
 * restated so the tests check its codes and its search against the oracle. */
int vo_u8_grid(const float* vecs, int64_t n, int dim, float* lo, float* s, float* inv) {
    int    affine = 0;
    float* hi     = (float*)malloc(sizeof(float) * (size_t)dim);
    for (int d = 0; d < dim; ++d) {
        lo[d] = INFINITY;
        hi[d] = -INFINITY;
    }
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) {
            const float x = vecs[(size_t)i * dim + d];
            if (x < lo[d]) lo[d] = x;
            if (x > hi[d]) hi[d] = x;
            if (!(x >= 0.f && x <= 255.f && rintf(x) == x)) affine = 1;
        }
    float range = 0.f;
    for (int d = 0; d < dim; ++d) {
        const float r = hi[d] - lo[d];
        if (r > range) range = r;
    }
    free(hi);
    if (!affine) {
        for (int d = 0; d < dim; ++d) lo[d] = 0.f;
        *s   = 1.f;
        *inv = 1.f;
        return 0;
    }
    *s   = range > 0.f ? range / 255.f : 1.f;
    *inv = 1.f / *s;
    return 1;
}

void vo_u8_codes(const float* x, int64_t n, int dim, const float* lo, float inv, uint8_t* out) {
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) {
            const float v = x[(size_t)i * dim + d];
            float       c = lo ? rintf((v - lo[d]) * inv) : rintf(v);
            c             = c < 0.f ? 0.f : (c > 255.f ? 255.f : c);
            out[(size_t)i * dim + d] = (uint8_t)c;
        }
}

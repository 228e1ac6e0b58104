/*
 * vann_oracle.h -- CPU restatement of the reference's Vamana / FreshVamana hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * product in cs5013-project_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * never calls it and has no CPU fallback.
 *
 * Each function cites the reference code it restates (paths relative to the
 * reference project root).  Where the reference is non-deterministic (atomic
 * arrival order, racy bloom-filter check-then-set), the oracle fixes one member
 * of the reference's allowed behaviour set and the CUDA kernels implement the
 * same member:
 *   - bloom filter: adjacency slots are processed in chunks of 32 in adjacency
 *     order; every slot of a chunk is checked against the filter as it stood
 *     before the chunk, then the chunk's new neighbours are marked.  This is
 *     what one convergent warp of filterNeighbors (vamana/include/search.cuh:119-137)
 *     does.  VO_BLOOM_SEQUENTIAL (chunk 1) and VO_BLOOM_SNAPSHOT (whole list)
 *     are the two other members, kept for the golden-graph experiment.
 *   - new neighbours of one expansion with equal distance are ordered by node id
 *     (the reference orders them by atomicAdd arrival, search.cuh:134).
 *   - reverse-index entries arrive in ascending source-node order, each source's
 *     entries in RobustPrune selection order (kernels.cuh:293-301 uses atomics).
 */
#ifndef VANN_ORACLE_H
#define VANN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VO_BF_ENTRIES 39988u /* vamana/include/bloom_filter.cuh:7 */
#define VO_NONE 0xFFFFFFFFu

enum { VO_BLOOM_CHUNK32 = 0, VO_BLOOM_SEQUENTIAL = 1, VO_BLOOM_SNAPSHOT = 2 };

/* status codes (match include/vann.h) */
enum { VO_OK = 0, VO_ERR_INVALID = 1, VO_ERR_HOP_LIMIT = 5 };

typedef struct {
    const float*    vecs;  /* n x dim, row-major */
    int64_t         n;
    int32_t         dim;
    uint32_t*       deg;   /* n */
    uint32_t*       adj;   /* n x R */
    int32_t         R;
    const uint32_t* tomb;  /* bitmap of deleted ids (bit i of word i>>5), may be NULL */
} vo_graph;

uint32_t vo_bf_h1(uint32_t x);
uint32_t vo_bf_h2(uint32_t x);
float    vo_l2sq(const float* a, const float* b, int dim);

/* One GreedySearch (vamana/include/search.cuh:20-367).
 * Outputs the final worklist (<= L entries, sorted) and the expansion list
 * (parents in expansion order, capped at max_visited) with their distances. */
int vo_search_one(const vo_graph* g, const float* q, int L, uint32_t entry, uint32_t skip_id,
                  int bloom_mode, int max_visited, int max_hops, uint32_t* wl_ids, float* wl_d,
                  int* wl_n, uint32_t* vis_ids, float* vis_d, int* vis_n, int* hops,
                  int64_t* evals, int64_t* adjw);

/* Batched search: out_ids/out_d are n x k (padded with VO_NONE / +inf).
 * skip_mode: 0 = no skip, 1 = skip the query's batch index (reference quirk
 * search.cuh:126).  hops/evals/adjw may be NULL; adjw counts the adjacency words
 * read (the sum of the expanded parents' degrees).  threads <= 0 means all cores. */
int vo_search_batch(const vo_graph* g, const float* q, int64_t nq, int L, int k, uint32_t entry,
                    int skip_mode, int bloom_mode, int max_hops, uint32_t* out_ids, float* out_d,
                    int32_t* hops, int64_t* evals, int64_t* adjw, int threads);

/* RobustPrune over a sorted candidate list (kernels.cuh:232-356).  Returns the
 * new degree; writes the chosen ids in selection order to out. */
int vo_robust_prune(const vo_graph* g, const float* node_vec, const uint32_t* cand,
                    const float* cand_d, int nc, float alpha, int R, uint32_t* out,
                    int64_t* evals);

/* One Vamana batch (vamana_impl.cuh:289-360 runVamana / :182-265 patchGraph):
 * search every batch node from `entry`, RobustPrune its out-neighbours,
 * record reverse edges, then re-prune every node 0..n-1 over reverse u out.
 * Batch nodes are ids batch_start .. batch_start+batch_n-1 and their vectors are
 * g->vecs rows.  skip_mode: 0 none, 1 batch index (reference), 2 node id.
 * g->deg / g->adj are updated in place. */
int vo_vamana_batch(vo_graph* g, int64_t batch_start, int64_t batch_n, int L, float alpha,
                    uint32_t entry, int max_visited, int max_reverse, int skip_mode,
                    int bloom_mode, int threads);

/* FreshVamana delete consolidation (FreshDiskANN, Singh et al. 2021, Algorithm 4)
 * over the ids marked in g->tomb; the candidate order is fixed as described in
 * vann_oracle.c.  g->deg / g->adj are updated in place; the ids freed by this call
 * (deleted and not marked in is_free) are written ascending to `freed` (n entries
 * at most) and counted in n_freed; new_entry is the entry point afterwards. */
int vo_consolidate(vo_graph* g, float alpha, int cap, const unsigned char* is_free, uint32_t entry,
                   uint32_t* new_entry, uint32_t* freed, int64_t* n_freed, int threads);

/* The same batch over the node ids nodes[0 .. batch_n) in that order (inserts into ids
 * freed by a consolidation, taken from the free list): queries are those nodes' rows
 * in g->vecs; reverse entries reach each target in batch order. */
int vo_vamana_batch_ids(vo_graph* g, const uint32_t* nodes, int64_t batch_n, int L, float alpha,
                        uint32_t entry, int max_visited, int max_reverse, int skip_mode, int bloom_mode,
                        int threads);

/* Deterministic random initial graph (hash-based, no self loops). */
void vo_random_graph(int64_t n, int R, uint64_t seed, uint32_t* deg, uint32_t* adj);

/* argmin_i ||x_i - mean||^2 in FP64 (parth/tools/vamana.py:25-29). */
int64_t vo_medoid(const float* vecs, int64_t n, int dim);

/* Exact kNN in FP64 (ties by id). */
/* searchPoints2's merge (vamana/include/utils.cuh:199-285 merge_and_rerank_kernel,
 * distances as l2_distance_sq :150-158): for each query, the L graph worklist ids
 * then the n_il insert-list rows compete for L slots in that order.  A candidate
 * enters when its squared distance is strictly below the largest slot value and
 * replaces the first slot holding that value; the slots start at +inf.  The slots
 * are then bubble-sorted by distance.  Graph candidates are reported by id, insert-
 * list row s as 0x80000000 | s; unfilled slots as 0xFFFFFFFF with +inf. */
void vo_merge_rerank(const float* vecs, int dim, const float* q, int64_t nq, const uint32_t* graph_ids,
                     int L, const float* insert_list, int64_t n_il, uint32_t* out_ids, float* out_d);

void vo_bruteforce_knn(const float* base, int64_t n, const float* q, int64_t nq, int dim, int k,
                       uint32_t* out_ids, double* out_d, int threads);

/* The uint8 traversal copy of float rows (no counterpart in the reference: a
 * reduced-precision form beside it).  The grid fitted to rows 0 .. n-1: when every
 * value is an integer in [0, 255] the identity (returns 0; lo = 0, s = inv = 1), else
 * (returns 1) lo[d] = the column minimum and one scale s = max_d (max_d - lo[d]) / 255
 * (1 when every column is constant), inv = 1 / s, all in FP32. */
int vo_u8_grid(const float* vecs, int64_t n, int dim, float* lo, float* s, float* inv);
/* Codes of n rows (or queries) on a grid: rint((x - lo[d]) * inv) clamped to [0, 255]
 * (round half to even); lo NULL: the identity grid, rint(x) clamped. */
void vo_u8_codes(const float* x, int64_t n, int dim, const float* lo, float inv, uint8_t* out);

#ifdef __cplusplus
}
#endif
#endif

// kernels.h -- launch interfaces of the CUDA kernels (host <-> device boundary
// inside libvann.so; the public C ABI is include/vann.h).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace vann {

// message for vann_last_error() on this host thread
void set_last_error(const char* msg);

struct SearchArgs {
    const void*     store;     // traversal copy (F32 / BF16 / FP8 / U8 rows)
    const float2*   scale;     // FP8 copy: per row (scale, scale^2 * |codes|^2)
    const float*    center;    // FP8 copy: per-dimension centre the codes are relative to
    const float*    pq_cb;     // PQ copy: [D / 8][256][8] centroids
    const float*    pq_cnorm;  // PQ copy: [D / 8] largest centroid norm per subspace
    const float*    vecs_f32;  // exact rows (rerank)
    const uint32_t* deg;
    const uint32_t* adj;
    const uint32_t* adj_h;     // packed filter slots of every adjacency entry
    uint32_t        R;
    const uint32_t* tomb;      // tombstone bitmap or null
    const float*    queries;   // nq x D FP32
    uint64_t        nq;
    uint32_t        D;
    uint32_t        L, k, entry, max_hops;   // L, k: the launch's maxima
    const uint32_t* Lq;        // per-query worklist size (<= L) or null
    const uint32_t* kq;        // per-query result count (<= k) or null
    uint32_t        skip_mode;  // 0 none, 1 batch index, 2 skip_base + batch index
    uint32_t        skip_base;
    uint32_t        beam;       // parents expanded per hop: 0/1 (the reference's search) or 2
    int             int_queries; // every query is a row of the exact uint8 copy (build / insert)
    int             rerank;
    uint32_t*       out_ids;    // nq x k or null
    float*          out_d;
    uint32_t*       vis_ids;    // nq x max_visited expansion lists or null
    float*          vis_d;
    uint32_t*       vis_n;
    uint32_t        max_visited;
    uint32_t*       hops_out;   // per-query hop / distance-evaluation counts or null
    uint32_t*       evals_out;
    uint32_t*       adjw_out;   // per-query adjacency words read (sum of parent degrees)
    const uint32_t* order;      // order in which warps take the queries (a permutation) or null
    uint32_t*       counter;    // zeroed before launch (by the order kernel when there is one)
    int             pdl;        // launched as a programmatic dependent of the order kernel
    uint32_t*       status;
};

cudaError_t launch_search(const SearchArgs& a, int store, int num_sms, cudaStream_t st, int variant = 0);
int         search_variants();

// RobustPrune over candidates A (expansion list or reverse entries) merged with
// B (the node's current out-neighbours).
struct PruneArgs {
    const float*    vecs;      // FP32 rows
    uint32_t        D;
    uint32_t*       deg;
    uint32_t*       adj;
    uint32_t*       adj_h;     // packed filter slots, rewritten with adj
    uint32_t        R;
    float           alpha;
    uint32_t        cap;       // merged-list cap (max_visited or max_reverse)
    // nodes to prune: node_ids[i] for i < n_nodes, or all ids < n_nodes when null
    const uint32_t* node_ids;
    uint64_t        n_nodes;
    // A as per-node lists (out-prune): a_ids/a_d [n_nodes x a_stride], a_n;
    // a_d null: the distances to the node are computed here
    const uint32_t* a_ids;
    const float*    a_d;
    const uint32_t* a_n;
    uint32_t        a_stride;
    // A as CSR of reverse sources (re-prune): sources of node v in
    // csr_src[csr_off[v] .. csr_off[v] + csr_cnt[v]) sorted ascending
    const uint32_t* csr_off;
    const uint32_t* csr_cnt;
    const uint32_t* csr_src;
    int             csr_by_slot; // csr_off / csr_cnt indexed by position in node_ids, not by id
    int             use_b;       // include the node's current out-neighbours
    int             skip_empty;  // re-prune: skip nodes without reverse entries
    int             consistent;  // B lists are alpha-consistent: skip B-B checks
    uint32_t*       counter;     // work counter, zeroed before launch
    uint32_t*       status;
    // tensor-core passes (prune_tc.cu) and the hand-off between kernels
    const uint8_t*  vecs_u8;     // exact uint8 rows (or null)
    const uint32_t* gate;        // non-zero: the uint8 rows are not exact
    const uint32_t* in_list;     // prune_kernel: only the slots in_list[0 .. *in_count) (when set)
    const uint32_t* in_count;
    unsigned long long* pruned;  // [0] tensor-core, [1] CUDA-core node counts (or null)
};

// prune_kernel: every node, or the listed slots when a.in_count is set.
cudaError_t launch_prune(const PruneArgs& a, int num_sms, cudaStream_t st);
bool        prune_tc_supported(uint32_t D, uint32_t R);
// Tensor-core passes over in_list (every node when null); leftovers to out_list.
// ws: 2 * n_nodes + 4 words of scratch; counters: three zeroed work counters.
cudaError_t launch_prune_tc(const PruneArgs& a, const uint32_t* in_list, const uint32_t* in_count,
                            uint32_t* out_list, uint32_t* out_count, uint32_t* ws, uint32_t* counters, int num_sms,
                            cudaStream_t st);
// Reverse re-prune of consistent lists, one warp per node (prune_rev.cu): nodes
// with more than 128 candidates or 8 reverse sources are handed on in out_list.
// u8: distances from a.vecs_u8 (the host has read that every row is exact).
cudaError_t launch_prune_rev(const PruneArgs& a, bool u8, uint32_t* out_list, uint32_t* out_count, int num_sms,
                             cudaStream_t st);

// searchPoints2's merge of graph results with the insert list (staged.cu)
struct StagedArgs {
    const float*    queries;    // nq x D
    uint64_t        nq;
    const float*    vecs;       // graph rows
    const uint32_t* graph_ids;  // nq x L worklist entries (kNone: padding)
    uint32_t        L, D;
    const float*    stage;      // n_stage x D insert-list rows
    uint64_t        n_stage;
    uint32_t*       out_ids;    // nq x L: graph id, or 0x80000000 | insert-list row
    float*          out_d;      // nq x L
    float*          out_vecs;   // nq x L x D or null
    uint32_t        p2;         // set by the launcher
};
cudaError_t launch_staged_merge(const StagedArgs& a, int num_sms, cudaStream_t st);

// graph utilities (graph_ops.cu)
cudaError_t launch_random_graph(uint32_t* deg, uint32_t* adj, uint32_t* adj_h, uint64_t first,
                                uint64_t n, uint32_t R, uint64_t seed, cudaStream_t st);
cudaError_t launch_hash_rows(const uint32_t* adj, uint32_t* adj_h, uint64_t n, uint32_t R,
                             cudaStream_t st);
// inexact: set non-zero when a uint8 code is not exactly its FP32 value
// FP8: the codes encode row - center[] with scale[row] = (s, s^2 * |codes|^2),
// s = amax / 448 of the centred row.  uint8: center = the fitted grid's offsets and
// inv its 1 / scale (launch_u8_grid), or nullptr for the identity grid.
cudaError_t launch_convert(const float* src, void* dst, float2* scale, const float* center, float inv,
                           uint64_t rows, uint32_t D, int store, uint32_t* inexact, cudaStream_t st);
cudaError_t launch_convert_ids(const float* vecs, const uint32_t* ids, uint64_t n, void* dst, float2* scale,
                               const float* center, float inv, uint32_t D, int store, uint32_t* inexact,
                               cudaStream_t st);
// The uint8 copy's grid fitted to rows 0 .. n-1: lo[D] offsets and grid[3] =
// {affine flag, scale, 1 / scale}; the identity (lo 0, scale 1, flag 0) when every
// value is an integer in [0, 255].  ws: u8_grid_ws_bytes(D).
size_t      u8_grid_ws_bytes(uint32_t D);
cudaError_t launch_u8_grid(const float* vecs, uint64_t n, uint32_t D, void* ws, float* lo, float* grid,
                           cudaStream_t st);

// Searches over a uint8 copy on a fitted grid (rerank.cu).  The queries are mapped onto
// the grid first -- round((q - lo) / s) clamped to [0, 255], an integer-valued FP32 copy
// -- so the search kernels run their exact integer path on code distances; the result
// is then either reranked from the exact FP32 rows or its distances scaled by s^2.
cudaError_t launch_grid_queries(const float* q, uint64_t nq, uint32_t D, const float* lo, float inv, float* out,
                                cudaStream_t st);
// Exact FP32 rerank of per-query candidate lists: cand [nq][L] in worklist order
// (kNone past the list's end) -> the k closest by (exact distance, list position),
// per-query counts kq (or null: k for all); the rerank the search kernels apply
// in-kernel, as a separate pass.
cudaError_t launch_rerank(const float* vecs, const float* q, uint64_t nq, uint32_t D, const uint32_t* cand,
                          uint32_t L, const uint32_t* kq, uint32_t k, uint32_t* out_ids, float* out_d,
                          int num_sms, cudaStream_t st);
cudaError_t launch_scale(float* x, uint64_t n, float f, cudaStream_t st);
// float bits of each column's largest magnitude over rows 0 .. n-1
cudaError_t launch_col_bounds(const float* vecs, uint64_t n, uint32_t D, uint32_t* bound, cudaStream_t st);
// PQ codebook (pq.cu): cb [D / 8][256][8] centroids trained on rows 0 .. n-1, cnorm [D / 8]
// largest centroid norm per subspace; ws: pq_train_ws_bytes(n, D).  D % 128 == 0.
size_t      pq_train_ws_bytes(uint64_t n, uint32_t D);
cudaError_t launch_pq_train(const float* vecs, uint64_t n, uint32_t D, float* cb, float* cnorm, void* ws,
                            cudaStream_t st);
// codes [row][D / 8] of rows first .. first + rows - 1, or of rows ids[0 .. rows) when ids is set
cudaError_t launch_pq_encode(const float* vecs, uint64_t first, uint64_t rows, const uint32_t* ids, uint32_t D,
                             const float* cb, uint8_t* codes, cudaStream_t st);
// FP32 column means of rows 0 .. n-1 (the medoid's exact column sums); ws: medoid_ws_bytes(D)
cudaError_t launch_col_mean(const float* vecs, uint64_t n, uint32_t D, void* ws, float* mean, cudaStream_t st);
cudaError_t launch_iota(uint32_t* out, uint64_t n, uint32_t first, cudaStream_t st);
cudaError_t launch_set_bits(uint32_t* bits, const uint32_t* ids, uint64_t n, uint64_t limit,
                            cudaStream_t st);
// Medoid of rows 0 .. n-1 into ws (medoid_ws_bytes(D) bytes); the id ends in
// medoid_best(ws, D)[1] and, when d_out is set, in *d_out.  Allocates nothing.
size_t              medoid_ws_bytes(uint32_t D);
unsigned long long* medoid_best(void* ws, uint32_t D);
cudaError_t launch_medoid(const float* vecs, uint64_t n, uint32_t D, void* ws, uint32_t* d_out, cudaStream_t st);
cudaError_t launch_edges(const uint32_t* nodes, uint64_t n_nodes, const uint32_t* deg,
                         const uint32_t* adj, uint32_t R, uint32_t* keys, uint32_t* vals,
                         uint32_t* counts, cudaStream_t st);
cudaError_t launch_find_vectors(const float* vecs, uint64_t n, uint32_t D, const float* q,
                                uint64_t nq, const uint32_t* tomb, int32_t* out, cudaStream_t st);
// candidate lists of the live nodes first .. first+n-1 that have a deleted neighbour
cudaError_t launch_consolidate_candidates(const uint32_t* deg, const uint32_t* adj, uint32_t R,
                                          const uint32_t* tomb, uint64_t first, uint64_t n, uint32_t* node_list,
                                          uint32_t* n_list, uint32_t* cand, uint32_t* cand_n, uint32_t cap,
                                          int num_sms, cudaStream_t st);

}  // namespace vann

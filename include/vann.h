/*
 * vann.h -- C ABI of the B200-native Vamana / FreshVamana engine (libvann.so).
 *
 * Every entry point takes plain pointers and sizes, returns a vann_status and
 * never exits the process.  Device pointers are caller-owned CUDA device memory
 * on the current device; `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream).  One vann_index is externally synchronised: do not
 * call into the same handle from two host threads at once.
 *
 * The reference interface each entry point replaces is cited beside it
 * (paths relative to the reference project, VishankSingh/CS5013-Project).
 */
#ifndef VANN_H
#define VANN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: vann_search_params gained `beam` (a caller built against 1 passes a shorter struct) */
#define VANN_ABI_VERSION 2

typedef enum {
    VANN_OK              = 0,
    VANN_ERR_INVALID     = 1,  /* bad argument */
    VANN_ERR_CUDA        = 2,  /* a CUDA runtime call failed (see vann_last_error) */
    VANN_ERR_CAPACITY    = 3,  /* index capacity exhausted */
    VANN_ERR_IO          = 4,  /* file could not be read or written */
    VANN_ERR_HOP_LIMIT   = 5,  /* a search stopped at max_hops (results are still written) */
    VANN_ERR_NOT_FOUND   = 6,  /* delete-by-vector found no matching node */
    VANN_ERR_TIMEOUT     = 7,  /* a bounded device wait gave up */
    VANN_ERR_OOM         = 8,  /* device allocation failed */
    VANN_ERR_UNSUPPORTED = 9,  /* combination not built (e.g. dim not a multiple of 4) */
    VANN_ERR_STATE       = 10  /* call not valid in the index's current state */
} vann_status;

/* Storage forms of the base vectors.  F32 is always kept (exact distances,
 * pruning, rerank); the others are extra traversal copies. */
typedef enum {
    VANN_STORE_F32  = 0,
    VANN_STORE_BF16 = 1, /* round-to-nearest-even bf16, FP32 accumulation */
    VANN_STORE_FP8  = 2, /* e4m3 with one FP32 scale per vector (amax / 448) */
    VANN_STORE_U8   = 3, /* uint8 codes on a grid fitted to the rows that fill the
                            index (build / set / load): the identity, so the copy is
                            exact, when every value is an integer in [0, 255]; else
                            one offset per dimension (its minimum) and one scale
                            (the largest range / 255), queries rounded onto the same
                            grid, returned distances scaled back (approximate: meant
                            for rerank = 1).  Later inserts keep the grid. */
    VANN_STORE_PQ   = 4  /* product-quantized codes: one byte per 8 dimensions (256
                            k-means centroids per subspace), distances from a per-query
                            table; approximate, meant for rerank = 1; dim a multiple
                            of 128 (BANG's compressed traversal, bang_exact/src/
                            parANN.cu:1107-1157) */
} vann_store;

/* Reference quirks, reproduced for parity when set. */
#define VANN_QUIRK_SKIP_BATCH_INDEX 0x1u /* skip neighbour id == query's batch index
                                            (vamana/include/search.cuh:126) */

typedef struct {
    uint32_t dim;         /* D; must be a multiple of 4, <= 512 */
    uint32_t degree;      /* R (max out-degree), <= 128 */
    uint32_t build_L;     /* worklist size used by build / insert searches */
    float    alpha;       /* RobustPrune alpha (reference hard-codes 1.5,
                             vamana/include/vamana_impl.cuh:297) */
    uint64_t capacity;    /* max number of nodes the index can hold */
    uint32_t max_visited; /* expansion-list cap per build search (reference 600,
                             vamana/include/constants.cuh:13) */
    uint32_t max_reverse; /* reverse-candidate cap per node (reference 500,
                             vamana/include/constants.cuh:20) */
    uint32_t flags;       /* VANN_QUIRK_* applied to build / insert searches */
    uint32_t stores;      /* bitmask (1 << vann_store) of extra traversal copies */
} vann_params;

typedef struct {
    uint32_t L;        /* worklist size, >= k, <= 1024 */
    uint32_t k;        /* results per query */
    uint32_t store;    /* vann_store the traversal reads */
    uint32_t rerank;   /* 1: exact FP32 rerank of the final worklist before top-k */
    uint32_t flags;    /* VANN_QUIRK_* */
    uint32_t max_hops; /* 0 = default (1,000,000) */
    uint32_t beam;     /* parents expanded per hop: 0 or 1 = the reference's GreedySearch
                          (search.cuh:226-367, one parent per iteration); 2 = the first
                          two unvisited entries together (a batched form with its own
                          results, not the reference's; needs L <= 64, dim <= 128,
                          degree <= 64, else VANN_ERR_UNSUPPORTED) */
} vann_search_params;

typedef struct {
    uint64_t size;         /* node ids in use (0 .. size-1, some may be deleted) */
    uint64_t capacity;
    uint64_t live;         /* size minus deleted */
    uint64_t free_ids;     /* consolidated ids waiting for reuse */
    uint32_t entry;        /* search entry point */
    uint32_t dim, degree;
    uint32_t consistent;   /* 1 when every adjacency list came from RobustPrune with alpha */
    uint64_t device_bytes; /* device memory held by the index */
    uint64_t pruned_tc;    /* RobustPrune runs done with the Gram matrix on the tensor cores */
    uint64_t pruned_cuda;  /* RobustPrune runs done on the CUDA cores (float rows, overflow) */
    uint64_t staged;       /* rows in the insert list (vann_stage_insert), not yet in the graph */
} vann_info;

typedef struct vann_index vann_index;

const char* vann_status_string(vann_status s);
/* Message of the last failing call on this host thread ("" if none). */
const char* vann_last_error(void);
int         vann_abi_version(void);

/* Vamana<T>::Vamana storage + GraphT (vamana/include/vamana.cuh:36-146,
 * graphT.cuh:56-59).  Allocates capacity on the current device. */
vann_status vann_create(const vann_params* params, vann_index** out);
vann_status vann_destroy(vann_index* index);
vann_status vann_get_info(const vann_index* index, vann_info* out);

/* initGraph (vamana/include/utils.cuh:113-148): read n records of
 * {float vec[D]; uint32 deg; uint32 nbr[R]} (772 bytes at D=128, R=64). */
vann_status vann_load_graph(vann_index* index, const char* path, uint64_t n, uint32_t entry);
/* saveGraph (vamana.cu:1346-1362): write size records in the same layout. */
vann_status vann_save_graph(vann_index* index, const char* path);

/* Host-array graph upload / download (test and interop path).  consistent=1
 * asserts that every list came from RobustPrune with this index's alpha, as a set:
 * later batches then re-prune only the nodes that receive new edges (the reference
 * re-prunes every node, which for such a list gives back the same set in RobustPrune
 * order; a list held in another order keeps that order until it is touched). */
vann_status vann_set_graph(vann_index* index, const float* h_vecs, const uint32_t* h_deg,
                           const uint32_t* h_adj, uint64_t n, uint32_t entry, uint32_t consistent);
vann_status vann_get_graph(vann_index* index, float* h_vecs, uint32_t* h_deg, uint32_t* h_adj);

/* Vamana<T>::Vamana -> runVamana (vamana/include/vamana_impl.cuh:10-20,289-360).
 * Builds over n device vectors.  batch >= n: one batch over a seeded random
 * R-regular start graph (the reference build).  batch < n: that build on the
 * first batch, then batched inserts of `batch` nodes.  entry = UINT32_MAX picks
 * the medoid (argmin distance to the centroid) of the first batch.
 * Synchronises `stream` before returning. */
vann_status vann_build(vann_index* index, const float* d_vecs, uint64_t n, uint64_t batch,
                       uint64_t seed, uint32_t entry, void* stream);

/* runVamana over the graph already in the index (vann_load_graph /
 * vann_set_graph): the loaded adjacency is the start graph, exactly as the
 * reference builds over the random graph it reads (vamana_impl.cuh:289-360,
 * utils.cuh:113-148).  One batch over every node.  Synchronises `stream`. */
vann_status vann_build_loaded(vann_index* index, void* stream);

/* Vamana<T>::searchPoints (vamana/include/vamana_impl.cuh:55-96, GreedySearch
 * search.cuh:226-367).  d_queries: nq x dim FP32.  Writes nq x k ids / squared
 * L2 distances, padded with UINT32_MAX / +inf.  Asynchronous on `stream`. */
vann_status vann_search(vann_index* index, const float* d_queries, uint64_t nq,
                        const vann_search_params* sp, uint32_t* d_ids, float* d_dists,
                        void* stream);
/* vann_search plus per-query work counters (device arrays of nq, any may be
 * NULL): expansions (hops), distance evaluations, adjacency words read. */
vann_status vann_search_stats(vann_index* index, const float* d_queries, uint64_t nq,
                              const vann_search_params* sp, uint32_t* d_ids, float* d_dists,
                              uint32_t* d_hops, uint32_t* d_evals, uint32_t* d_adj_words,
                              void* stream);
/* Autotuner: times every compiled launch variant of the search kernel for this
 * (store, rerank, L) on the given queries (device time, CUDA events on
 * `stream`) and makes the fastest one the index's choice for later
 * vann_search calls with the same store, rerank and L.  Synchronises. */
vann_status vann_autotune(vann_index* index, const float* d_queries, uint64_t nq,
                          const vann_search_params* sp, float* h_ms_out, void* stream);
/* Number of compiled search variants (length of vann_autotune's h_ms_out,
 * which may be NULL; it receives the mean ms of each variant). */
int vann_search_variant_count(void);
/* vann_search over a batch whose queries have their own worklist size and result
 * count: d_L[i] <= sp->L and d_k[i] <= sp->k (device arrays of nq; sp->L, sp->k
 * are the batch maxima and size the launch).  Row i of d_ids / d_dists has
 * stride sp->k and is padded past d_k[i] with UINT32_MAX / +inf.  One launch
 * serves the whole uneven batch.  Asynchronous on `stream`. */
vann_status vann_search_uneven(vann_index* index, const float* d_queries, uint64_t nq,
                               const vann_search_params* sp, const uint32_t* d_L, const uint32_t* d_k,
                               uint32_t* d_ids, float* d_dists, void* stream);
/* Device status word of earlier asynchronous calls: synchronises `stream`,
 * returns VANN_ERR_HOP_LIMIT if a search hit its hop cap since the last call,
 * and clears it. */
vann_status vann_sync(vann_index* index, void* stream);

/* Vamana<T>::insertPoints + patchGraph (vamana_impl.cuh:22-33,182-265):
 * inserts n device vectors as one batch (search, RobustPrune, reverse edges,
 * re-prune of the touched nodes).  New ids (reused consolidated ids first,
 * then appended) go to d_ids_out (may be NULL).  Synchronises `stream`. */
vann_status vann_insert(vann_index* index, const float* d_vecs, uint64_t n, uint32_t* d_ids_out,
                        void* stream);

/* Vamana<T>::deletePoints (vamana_impl.cuh:35-53) by id: lazy tombstones that
 * searches skip (delete_list.cuh:109-115).  Asynchronous. */
vann_status vann_delete(vann_index* index, const uint32_t* d_ids, uint64_t n, void* stream);
/* deletePoints by exact vector match (findPointsKernel, kernels.cuh:905-933).
 * d_ids_out[i] = matched id or -1.  Synchronises `stream`. */
vann_status vann_delete_by_vector(vann_index* index, const float* d_vecs, uint64_t n,
                                  int32_t* d_ids_out, void* stream);

/* Vamana<T>::patchGraph (vamana_impl.cuh:182-265) extended with FreshVamana
 * delete consolidation: every live node that points at a deleted node is
 * re-pruned over its live out-neighbours plus the deleted nodes' live
 * out-neighbours; deleted ids are then freed for reuse.  Synchronises. */
vann_status vann_consolidate(vann_index* index, void* stream);

/* Vamana<T>::insertPoints (vamana_impl.cuh:22-33; InsertList::addVectors,
 * insert_list.cuh:12-87): append n device rows (n x dim FP32) to the index's insert
 * list, outside the graph.  vann_search_staged sees them; vann_patch_graph moves
 * them into the graph.  Synchronises `stream`. */
vann_status vann_stage_insert(vann_index* index, const float* d_vecs, uint64_t n, void* stream);

/* Vamana<T>::searchPoints2 (vamana_impl.cuh:98-180, merge_and_rerank_kernel
 * utils.cuh:199-285): GreedySearch with worklist sp->L (sp->k is ignored), then the
 * L worklist entries followed by every insert-list row compete for L slots by FP32
 * squared distance, computed sequentially over the dimensions like l2_distance_sq
 * (utils.cuh:150-158).  A candidate enters when strictly closer than the farthest
 * slot and replaces the first slot at that distance; the slots are returned in
 * stable distance order.  Per query L entries: d_ids holds graph ids, or
 * VANN_STAGED_ID(s) for insert-list row s (0xFFFFFFFF for an unfilled slot);
 * d_dists the distances; d_vecs_out (may be NULL) the rows themselves (nq x L x dim),
 * which is what searchPoints2 returns.  Asynchronous on `stream`. */
#define VANN_STAGED_ID(s) (0x80000000u | (uint32_t)(s))
vann_status vann_search_staged(vann_index* index, const float* d_queries, uint64_t nq,
                               const vann_search_params* sp, uint32_t* d_ids, float* d_dists,
                               float* d_vecs_out, void* stream);

/* On-disk interop (no counterpart call in the reference; its tooling does this in
 * scripts/bang-preprocess.py:37-72).  BANG / DiskANN disk layout from the
 * reference's 772-byte records: <prefix>_disk.bin holds one record per node
 * (dim x FP32 vector, u32 degree, the degree neighbour ids sorted ascending, then
 * the record's remaining slots unchanged); <prefix>_disk_metadata.bin holds u64
 * medoid, u64 record bytes, u32 data type (2 = float), u32 dim, u32 degree, u32 n.
 * Every node must have 1..degree neighbours (the script rejects others).
 * vann_convert_graph_file converts a 772-byte record file on the host (no GPU);
 * vann_save_graph_bang writes the index's graph (unused slots zero, as
 * vann_save_graph writes them) with its entry point as the medoid. */
vann_status vann_convert_graph_file(const char* in_path, uint64_t n, uint32_t dim, uint32_t degree,
                                    uint32_t medoid, const char* out_prefix);
vann_status vann_save_graph_bang(vann_index* index, const char* out_prefix);

/* Versioned full-state file (no counterpart in the reference): the graph (any dim
 * and degree), tombstones, ids waiting for reuse, entry point and the consistency
 * flag, so a FreshVamana index resumes exactly.  Layout, little-endian: "VANNIDX\0",
 * u32 version (1), u32 dim, u32 degree, u32 consistent, u64 size, u64 deleted,
 * u64 free count, u32 entry, u32 0, then size x dim FP32 rows, size u32 degrees,
 * size x degree u32 ids, ceil(size / 32) u32 tombstone words, free-count u32 ids.
 * vann_load_index needs the index's dim and degree to match and capacity >= size. */
vann_status vann_save_index(vann_index* index, const char* path);
vann_status vann_load_index(vann_index* index, const char* path);

/* The insert half of Vamana<T>::patchGraph (vamana_impl.cuh:182-265): every
 * insert-list row, in order, goes into the graph as one vann_insert batch and the
 * list is emptied.  d_ids_out (may be NULL) receives their graph ids.  Synchronises. */
vann_status vann_patch_graph(vann_index* index, uint32_t* d_ids_out, void* stream);

/* ---------------------------------------------------------------- serving loop
 * No counterpart in the reference, whose driver issues one call at a time on the
 * default stream (vamana.cu:1782-1895).  A server owns a worker thread over one
 * index.  Requests carry host data.  Searches queued while batch slots are busy
 * are admitted together into the next free slot as one uneven launch (own k
 * and L per request) with its copies on the slot's stream, so several batches
 * run at once (continuous batching).  By default writes keep their place in the
 * request order: each search sees exactly the writes submitted before it.  With
 * commit_interval_us > 0 writes are group-committed instead (see the field).  Slot
 * device memory is allocated at creation and capped by hbm_budget. */
typedef struct {
    uint32_t max_batch;   /* queries per admitted batch */
    uint32_t slots;       /* batches on the GPU at once (one stream each) */
    uint64_t hbm_budget;  /* device bytes for batch slots (0 = no cap); fewer slots if smaller */
    uint32_t max_k;       /* largest k a search may ask for */
    uint32_t store;       /* vann_store searches traverse */
    uint32_t rerank;      /* exact FP32 rerank */
    uint32_t commit_interval_us; /* 0: strict request order; > 0: group commit of writes at most
                                    this often, searches served at the last committed epoch */
} vann_server_params;

typedef struct {
    uint32_t slots;        /* slots admitted under the budget */
    uint64_t slot_bytes;   /* device bytes per slot */
    uint64_t batches, queries, writes, max_inflight, queued;
    uint64_t epoch;        /* writes applied so far */
} vann_server_stats;

typedef struct vann_server vann_server;

vann_status vann_server_create(vann_index* index, const vann_server_params* params, vann_server** out);
vann_status vann_server_destroy(vann_server* server);
/* n <= max_batch host queries (n x dim FP32), k <= max_k, k <= L <= 1024. */
vann_status vann_server_submit_search(vann_server* server, const float* h_queries, uint32_t n, uint32_t k,
                                      uint32_t L, uint64_t* ticket);
vann_status vann_server_submit_insert(vann_server* server, const float* h_vecs, uint32_t n, uint64_t* ticket);
vann_status vann_server_submit_delete(vann_server* server, const uint32_t* h_ids, uint32_t n, uint64_t* ticket);
vann_status vann_server_submit_consolidate(vann_server* server, uint64_t* ticket);
/* Blocks until the request is done (timeout_ms 0 = 10 minutes).  Search: n x k ids
 * and distances; insert: the n new ids in h_ids.  latency_us: submit to done.
 * epoch: for a search, the number of writes it saw; for a write, its position in
 * the order writes were applied (1-based).  Any out pointer may be NULL. */
vann_status vann_server_wait(vann_server* server, uint64_t ticket, uint32_t* h_ids, float* h_dists,
                             double* latency_us, uint64_t* epoch, uint32_t timeout_ms);
vann_status vann_server_get_stats(vann_server* server, vann_server_stats* out);

/* Allocation-free entry-point selection.  No counterpart in the reference.
 * Computes the medoid used as the search entry point (argmin over the n rows
 * of d_vecs of the FP64 squared distance to their mean, smallest id on ties --
 * the same value vann_build picks) into *d_medoid_out, without allocating any
 * device memory: its scratch is a fixed device array inside libvann.so
 * (48 KiB + 256 B, kept by every device that loads the library until exit).
 * For callers that cannot call cudaMalloc/cudaFree: processes whose device
 * memory is owned by another allocator under a fixed budget, threads on a
 * latency-critical path that must not take the allocator's locks or the device
 * synchronisation that cudaFree implies, and code that must not meet an
 * allocation failure at call time.
 * Limits: dim <= 4096 (larger returns VANN_ERR_UNSUPPORTED), n < 2^32.
 * Asynchronous on `stream`.  The column sums are exact (fixed-point integer
 * sums), so the result does not depend on the order of the device's additions.
 * The first call on a device (and the first in a context created after a
 * cudaDeviceReset) resolves the array's device address; make it before any
 * stream capture.  A CUDA error already pending when the call is made is
 * reported (VANN_ERR_CUDA) and left pending.  Each device has one such array
 * and every call on that device shares it, keeping the previous call's contents
 * until the next call clears it: calls on one device that overlap on the GPU
 * (e.g. issued on different streams) race on it, so serialise them. */
vann_status vann_medoid_noalloc(const float* d_vecs, uint64_t n, uint32_t dim, uint32_t* d_medoid_out,
                                void* stream);

#ifdef __cplusplus
}
#endif
#endif

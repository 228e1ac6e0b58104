// index.cu -- host-side index object behind the C ABI (include/vann.h).
//
// Replaces the reference's Vamana<T> class and its GraphT / InsertList /
// DeleteList members (vamana/include/vamana.cuh:36-146, vamana_impl.cuh,
// insert_list.cuh, delete_list.cuh).  Differences by design: many indexes per
// process (no __managed__ globals), capacity allocated once (no realloc + copy
// per patch), every call stream-ordered and returning a status instead of
// exit(), structure-of-arrays storage with 64-bit offsets, and inserts that
// reach the graph in the same call.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <tuple>
#include <new>
#include <string>
#include <vector>

#include "../../include/vann.h"
#include "common.cuh"
#include "kernels.h"

namespace {

thread_local std::string g_last_error;

struct Fail {
    vann_status st;
};

void set_err(const std::string& m) { g_last_error = m; }

#define VCHECK(call)                                                                  \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            set_err(std::string(#call) + ": " + cudaGetErrorString(e_));              \
            throw Fail{e_ == cudaErrorMemoryAllocation ? VANN_ERR_OOM : VANN_ERR_CUDA}; \
        }                                                                             \
    } while (0)

#define VREQUIRE(cond, code, msg) \
    do {                          \
        if (!(cond)) {            \
            set_err(msg);         \
            throw Fail{code};     \
        }                         \
    } while (0)

// grow-only device buffer
struct DevBuf {
    void*  p     = nullptr;
    size_t bytes = 0;
    // Grows by at least half again, in 2 MiB steps: workspaces sized by batches of
    // slowly rising size (edge lists, sort scratch) are then reallocated a few times
    // instead of on every batch, and every cudaFree waits for the device.
    void ensure(size_t b) {
        if (b <= bytes) return;
        constexpr size_t kStep = size_t(2) << 20;
        size_t           want  = std::max(b, bytes + bytes / 2);
        want                   = (want + kStep - 1) / kStep * kStep;
        if (p) cudaFree(p);
        p     = nullptr;
        bytes = 0;
        VCHECK(cudaMalloc(&p, want));
        bytes = want;
    }
    template <typename T>
    T* as() const {
        return static_cast<T*>(p);
    }
    void release() {
        if (p) cudaFree(p);
        p     = nullptr;
        bytes = 0;
    }
};

// Squared FP32 distance from every query to the entry row (its float bits).
__global__ void entry_dist_kernel(const float* queries, uint64_t nq, uint32_t D, const float* entry_row,
                                  uint32_t* keys) {
    vann::grid_dependents_may_launch();  // the order kernel waits for the keys itself
    const uint64_t q    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31u;
    if (q >= nq) return;
    const float* row = queries + q * D;
    float        s   = 0.f;
    for (uint32_t i = lane; i < D; i += 32) {
        const float d = row[i] - entry_row[i];
        s             = fmaf(d, d, s);
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) keys[q] = __float_as_uint(s);
}

// One block orders the queries by distance to the entry point, farthest first, in
// kOrderBuckets equal-width distance buckets (order within a bucket is whatever the
// shared-memory atomics give: a schedule, not a result).  Two launches in all, where
// a device-wide radix sort of a 10k batch takes several.  It also zeroes the search's
// query counter (when given one), which saves the search a memset node; launched
// as a programmatic dependent of entry_dist_kernel, it starts while that kernel's
// last blocks run and waits for their keys, and lets the search's blocks start
// while it runs (they wait for it in turn).
constexpr int kOrderThreads = 1024;
constexpr int kOrderBuckets = 1024;
__global__ void __launch_bounds__(kOrderThreads) order_by_bucket_kernel(const uint32_t* keys, uint32_t nq,
                                                                        uint32_t* order, uint32_t* counter) {
    vann::grid_dependency_wait();
    vann::grid_dependents_may_launch();
    if (counter != nullptr && threadIdx.x == 0) *counter = 0u;
    __shared__ uint32_t cnt[kOrderBuckets];
    __shared__ float    lo_w[32], hi_w[32];
    const uint32_t t = threadIdx.x;
    float          lo = __int_as_float(0x7f800000), hi = 0.f;
    for (uint32_t i = t; i < nq; i += kOrderThreads) {
        const float d = __uint_as_float(keys[i]);
        lo = fminf(lo, d);
        hi = fmaxf(hi, d);
    }
    for (int o = 16; o; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((t & 31u) == 0) {
        lo_w[t >> 5] = lo;
        hi_w[t >> 5] = hi;
    }
    for (uint32_t b = t; b < kOrderBuckets; b += kOrderThreads) cnt[b] = 0;
    __syncthreads();
    lo = lo_w[0];
    hi = hi_w[0];
    for (int w = 1; w < kOrderThreads / 32; ++w) {
        lo = fminf(lo, lo_w[w]);
        hi = fmaxf(hi, hi_w[w]);
    }
    const float scale = hi > lo ? (float)kOrderBuckets / (hi - lo) : 0.f;
    auto bucket = [&](uint32_t i) {  // 0 holds the farthest queries
        const float x = (hi - __uint_as_float(keys[i])) * scale;
        return x >= (float)(kOrderBuckets - 1) ? (uint32_t)(kOrderBuckets - 1) : (x > 0.f ? (uint32_t)x : 0u);
    };
    for (uint32_t i = t; i < nq; i += kOrderThreads) atomicAdd(&cnt[bucket(i)], 1u);
    __syncthreads();
    {  // exclusive prefix over the buckets: one per thread, warp scans, then the warp totals
        static_assert(kOrderBuckets == kOrderThreads, "one bucket per thread");
        __shared__ uint32_t wsum[32];
        const uint32_t lane = t & 31u, w = t >> 5;
        const uint32_t c    = cnt[t];
        uint32_t       inc  = c;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += v;
        }
        if (lane == 31u) wsum[w] = inc;
        __syncthreads();
        if (w == 0) {
            uint32_t x = wsum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t v = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x += v;
            }
            wsum[lane] = x - wsum[lane];  // exclusive over the warps
        }
        __syncthreads();
        cnt[t] = wsum[w] + inc - c;
    }
    __syncthreads();
    for (uint32_t i = t; i < nq; i += kOrderThreads) order[atomicAdd(&cnt[bucket(i)], 1u)] = i;
}

__global__ void scatter_rows_kernel(const float* src, const uint32_t* ids, uint64_t n, uint32_t D,
                                    float* dst, uint32_t* deg, uint32_t* tomb) {
    uint64_t r    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (r >= n) return;
    uint32_t id = ids[r];
    for (uint32_t i = lane; i < D; i += 32) dst[(uint64_t)id * D + i] = src[r * D + i];
    if (lane == 0) {
        deg[id] = 0;
        atomicAnd(tomb + (id >> 5), ~(1u << (id & 31u)));
    }
}

__global__ void gather_rows_kernel(const float* src, const uint32_t* ids, uint64_t n, uint32_t D,
                                   float* dst) {
    uint64_t r    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (r >= n) return;
    uint32_t id = ids[r];
    for (uint32_t i = lane; i < D; i += 32) dst[r * D + i] = src[(uint64_t)id * D + i];
}

__global__ void clear_deg_kernel(const uint32_t* ids, uint64_t n, uint32_t* deg) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) deg[ids[i]] = 0;
}

constexpr int kCounterRing = 256;

}  // namespace

void vann::set_last_error(const char* msg) { set_err(msg); }

struct vann_index {
    vann_params p{};
    int         device  = 0;
    int         num_sms = 148;
    uint64_t    size    = 0;
    uint64_t    n_deleted = 0;  // tombstoned and not yet freed
    uint32_t    entry   = vann::kNone;
    bool        consistent = false;

    float*    vecs  = nullptr;
    void*     store[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // by vann_store
    float2*   fp8_scale = nullptr;  // per row (scale, scale^2 |codes|^2)
    float*    fp8_center = nullptr; // per dimension: the FP8 codes encode row - center
    float*    u8_lo = nullptr;      // uint8 copy: per-dimension offsets of its grid
    float*    u8_grid = nullptr;    // uint8 copy: {affine flag, scale, 1 / scale}
    bool      u8_affine = false;    // host copy of the grid: fitted (approximate) or identity
    float     u8_s = 1.f, u8_inv = 1.f;
    float*    pq_cb = nullptr;      // PQ copy: [D / 8][256][8] centroids
    float*    pq_cnorm = nullptr;   // PQ copy: [D / 8] largest centroid norm per subspace
    uint32_t* deg  = nullptr;
    uint32_t* adj  = nullptr;
    uint32_t* adj_h = nullptr;  // packed filter slots beside every adjacency entry
    uint32_t* tomb = nullptr;
    uint32_t* counters = nullptr;  // ring of work counters
    uint32_t* status   = nullptr;
    int       ring_pos = 0;
    size_t    held     = 0;

    std::vector<uint32_t> free_ids;  // consolidated ids, reused by inserts
    uint64_t stage_n = 0;  // rows in the insert list (stage), outside the graph
    // per-query L / k arrays of the vann_search_uneven call in progress
    const uint32_t* pending_Lq = nullptr;
    const uint32_t* pending_kq = nullptr;
    // launch-bound variant of the build and insert searches per row format (-1: not timed yet)
    int build_variant[4] = {-1, -1, -1, -1};
    // autotuned search variant per (store, rerank, beam, L)
    std::map<std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>, int> tuned;

    static uint32_t beam_of(const vann_search_params& sp) { return sp.beam == 2 ? 2u : 1u; }
    int variant_for(const vann_search_params& sp) const {
        auto it = tuned.find(std::make_tuple(sp.store, sp.rerank ? 1u : 0u, beam_of(sp), sp.L));
        return it == tuned.end() ? 0 : it->second;
    }

    // search order of large batches (distance keys, then the order), one workspace per
    // stream: searches in flight on different streams (the server's slots) never share it
    std::map<cudaStream_t, DevBuf> ord;
    // per stream, searches over the fitted uint8 grid: the queries on the grid and the
    // candidate lists of the rerank
    std::map<cudaStream_t, DevBuf> grid_ws;
    std::vector<void*>             ord_retired;  // outgrown order workspaces, freed at destroy
    DevBuf vis_ids, vis_d, vis_n, nodes, runs, ovf, stage, s2_ids, s2_d, e_keys, e_vals, e_keys2, e_vals2, counts, offsets, cub_tmp,
        medoid_ws, gather, cand, cand_n, list_n, out_tmp;

    void alloc(void** ptr, size_t bytes) {
        VCHECK(cudaMalloc(ptr, bytes));
        held += bytes;
    }
    ~vann_index() {
        cudaFree(vecs);
        for (void* s : store) cudaFree(s);
        cudaFree(fp8_scale);
        cudaFree(fp8_center);
        cudaFree(u8_lo);
        cudaFree(u8_grid);
        cudaFree(pq_cb);
        cudaFree(pq_cnorm);
        cudaFree(deg);
        cudaFree(adj);
        cudaFree(adj_h);
        cudaFree(tomb);
        cudaFree(counters);
        cudaFree(status);
        for (auto& o : ord) o.second.release();
        for (auto& o : grid_ws) o.second.release();
        for (void* r : ord_retired) cudaFree(r);
        for (DevBuf* b : {&vis_ids, &vis_d, &vis_n, &nodes, &runs, &ovf, &stage, &s2_ids, &s2_d, &e_keys, &e_vals, &e_keys2, &e_vals2,
                          &counts, &offsets, &cub_tmp, &medoid_ws, &gather, &cand, &cand_n,
                          &list_n, &out_tmp})
            b->release();
    }

    uint32_t* next_counter(cudaStream_t st, bool zero = true) {
        uint32_t* c = counters + (ring_pos++ % kCounterRing) * 32;
        if (zero) VCHECK(cudaMemsetAsync(c, 0, sizeof(uint32_t), st));
        return c;
    }

    uint64_t tomb_words() const { return (p.capacity + 31) / 32; }

    // Order in which the warps of a search launch take its queries, or null.  A batch
    // that outnumbers the resident warps ends with its slowest queries: warps take
    // the queries farthest from the entry point first, since those tend to take the
    // most hops and, started last, would run on alone.  The order only changes which
    // warp runs a query when, never its result.
    //
    // A search captured into a CUDA graph keeps the address of this workspace, so a
    // workspace that grows is retired (freed at vann_destroy), never freed while the
    // index lives; and a search issued while its stream is being captured allocates
    // nothing: when the stream's workspace is too small, that batch runs in input
    // order, with the same results.
    //
    // counter (optional): the search's query counter, zeroed by the order kernel; the
    // search may then be launched as its programmatic dependent (*pdl, false while the
    // stream is being captured: a captured search keeps plain stream order).
    const uint32_t* search_order(const float* d_queries, uint64_t nq, cudaStream_t st, uint32_t* counter = nullptr,
                                 bool* pdl = nullptr) {
        if (pdl) *pdl = false;
        if (nq <= 16ull * (uint64_t)num_sms || nq > 0x7FFFFFFFull) return nullptr;
        const size_t            need = sizeof(uint32_t) * 2 * nq;
        DevBuf&                 ob   = ord[st];
        cudaStreamCaptureStatus cs   = cudaStreamCaptureStatusNone;
        VCHECK(cudaStreamIsCapturing(st, &cs));
        const bool capturing = cs != cudaStreamCaptureStatusNone;
        if (ob.bytes < need) {
            if (capturing) return nullptr;
            if (ob.p) {
                ord_retired.push_back(ob.p);
                ob.p     = nullptr;
                ob.bytes = 0;
            }
            ob.ensure(need);
        }
        uint32_t* keys  = ob.as<uint32_t>();
        uint32_t* order = keys + nq;
        entry_dist_kernel<<<(unsigned)((nq + 7) / 8), 256, 0, st>>>(d_queries, nq, p.dim,
                                                                  vecs + (uint64_t)entry * p.dim, keys);
        VCHECK(cudaGetLastError());
        const bool chain = counter != nullptr && !capturing;
        VCHECK(vann::launch_kernel(order_by_bucket_kernel, dim3(1), dim3(kOrderThreads), 0, st, chain, keys,
                                   (uint32_t)nq, order, counter));
        if (pdl) *pdl = chain;
        return order;
    }

    uint32_t* u8_inexact() const { return status + vann::kWordU8Inexact; }
    int       u8_state = -1;  // exactness of the uint8 copy seen by the host: -1 unknown, 0 no, 1 yes

    // whether every row is exact in the uint8 copy (read from the device once after
    // the rows change)
    bool u8_exact(cudaStream_t st) {
        if (!store[3]) return false;
        if (u8_state < 0) {
            uint32_t f = 0;
            VCHECK(cudaMemcpyAsync(&f, u8_inexact(), sizeof(f), cudaMemcpyDeviceToHost, st));
            VCHECK(cudaStreamSynchronize(st));
            u8_state = f == 0u ? 1 : 0;
        }
        return u8_state == 1;
    }

    // the centre / offsets argument of the conversion kernels for traversal copy s
    const float* copy_center(int s) const {
        if (s == 2) return fp8_center;
        if (s == 3 && u8_affine) return u8_lo;
        return nullptr;
    }

    // rows [first, first + rows) -> traversal copies; rows from 0 replace every
    // row, so the uint8 exactness flag starts over and the FP8 centre (the rows'
    // column means) and the uint8 grid, both fixed until the rows are replaced
    // again, are recomputed
    void convert_rows(uint64_t first, uint64_t rows, cudaStream_t st) {
        u8_state = -1;
        if (first == 0) VCHECK(cudaMemsetAsync(u8_inexact(), 0, sizeof(uint32_t), st));
        if (first == 0 && store[2] && rows > 0) {
            medoid_ws.ensure(vann::medoid_ws_bytes(p.dim));
            VCHECK(vann::launch_col_mean(vecs, rows, p.dim, medoid_ws.p, fp8_center, st));
        }
        if (first == 0 && store[3] && rows > 0) {
            // the grid: identity for rows of integers in [0, 255], else fitted; the
            // host keeps a copy for the search launches
            medoid_ws.ensure(std::max(vann::medoid_ws_bytes(p.dim), vann::u8_grid_ws_bytes(p.dim)));
            VCHECK(vann::launch_u8_grid(vecs, rows, p.dim, medoid_ws.p, u8_lo, u8_grid, st));
            float g[3] = {0.f, 1.f, 1.f};
            VCHECK(cudaMemcpyAsync(g, u8_grid, sizeof(g), cudaMemcpyDeviceToHost, st));
            VCHECK(cudaStreamSynchronize(st));
            u8_affine = g[0] != 0.f;
            u8_s      = g[1];
            u8_inv    = g[2];
        }
        for (int s = 1; s < 4; ++s) {
            if (!store[s]) continue;
            size_t esz = s == 1 ? 2 : 1;
            void*  dst = static_cast<char*>(store[s]) + first * p.dim * esz;
            VCHECK(vann::launch_convert(vecs + first * p.dim, dst, s == 2 ? fp8_scale + first : nullptr,
                                        copy_center(s), u8_inv, rows, p.dim, s, u8_inexact(), st));
        }
        if (store[4] && rows > 0) {
            // PQ: the codebook is trained on the rows that replace every row, then fixed
            if (first == 0) {
                struct Scratch {  // training workspace, freed on every way out
                    DevBuf b;
                    ~Scratch() { b.release(); }
                } ws;
                ws.b.ensure(vann::pq_train_ws_bytes(rows, p.dim));
                VCHECK(vann::launch_pq_train(vecs, rows, p.dim, pq_cb, pq_cnorm, ws.b.p, st));
                VCHECK(cudaStreamSynchronize(st));  // before the workspace is freed
            }
            VCHECK(vann::launch_pq_encode(vecs, first, rows, nullptr, p.dim, pq_cb, static_cast<uint8_t*>(store[4]),
                                          st));
        }
    }

    // RobustPrune launch: the tensor-core pass when an exact uint8 copy exists
    // (decided on the device by the exactness flag), prune_kernel for the rest
    // RobustPrune launch.  Consistent reverse re-prunes go first to the warp-per-node
    // kernel; the tensor-core passes take what it hands on (or every node) when an
    // exact uint8 copy may exist (decided on the device by the exactness flag);
    // prune_kernel finishes whatever is left.
    void run_prune(vann::PruneArgs pa, cudaStream_t st) {
        if (pa.n_nodes == 0) return;
        pa.pruned = reinterpret_cast<unsigned long long*>(status + vann::kWordPruned);
        const uint64_t n   = pa.n_nodes;
        const bool     tc  = store[3] && vann::prune_tc_supported(p.dim, p.degree);
        const bool     rev = pa.consistent && pa.csr_off && pa.node_ids && p.dim <= 256;
        if (store[3]) {
            pa.vecs_u8 = static_cast<const uint8_t*>(store[3]);
            pa.gate    = u8_inexact();
        }
        // lists: [0, n] rev hand-off + count, [n+1, 2n+2) final hand-off + count, then tc scratch
        ovf.ensure(sizeof(uint32_t) * (4 * n + 8));
        uint32_t*       rev_list   = ovf.as<uint32_t>();
        uint32_t*       rev_count  = rev_list + n;
        uint32_t*       last_list  = rev_list + n + 1;
        uint32_t*       last_count = last_list + n;
        uint32_t*       ws         = last_count + 1;
        const uint32_t* in_list    = nullptr;  // every node
        const uint32_t* in_count   = nullptr;
        if (rev) {
            VCHECK(cudaMemsetAsync(rev_count, 0, sizeof(uint32_t), st));
            VCHECK(vann::launch_prune_rev(pa, u8_exact(st), rev_list, rev_count, num_sms, st));
            pa.counter = next_counter(st);
            in_list    = rev_list;
            in_count   = rev_count;
        }
        if (tc) {
            uint32_t* tc_counters = next_counter(st);  // one per pass
            VCHECK(cudaMemsetAsync(tc_counters + 1, 0, 2 * sizeof(uint32_t), st));
            VCHECK(vann::launch_prune_tc(pa, in_list, in_count, last_list, last_count, ws, tc_counters, num_sms,
                                         st));
            in_list  = last_list;
            in_count = last_count;
        }
        pa.in_list  = in_list;
        pa.in_count = in_count;
        VCHECK(vann::launch_prune(pa, num_sms, st));
    }

    // a bounded device wait that gave up is reported by the call that launched it
    void check_device_status() {
        uint32_t w = 0;
        VCHECK(cudaMemcpy(&w, status, sizeof(w), cudaMemcpyDeviceToHost));
        if (w & vann::kStatusTimeout) {
            VCHECK(cudaMemset(status, 0, sizeof(uint32_t)));
            VREQUIRE(false, VANN_ERR_TIMEOUT, "a bounded device wait gave up (tensor-core prune)");
        }
    }

    uint32_t medoid(uint64_t n, cudaStream_t st) {
        medoid_ws.ensure(vann::medoid_ws_bytes(p.dim));
        VCHECK(vann::launch_medoid(vecs, n, p.dim, medoid_ws.p, nullptr, st));
        unsigned long long hb[2];
        VCHECK(cudaMemcpyAsync(hb, vann::medoid_best(medoid_ws.p, p.dim), sizeof(hb), cudaMemcpyDeviceToHost, st));
        VCHECK(cudaStreamSynchronize(st));
        return (uint32_t)hb[1];
    }

    // One Vamana batch over the nodes in d_nodes (vectors already stored):
    // GreedySearch from the entry, out-prune, reverse edges, re-prune.
    void vamana_batch(const uint32_t* d_nodes, uint64_t count, const float* d_q, uint32_t skip_mode,
                      uint32_t skip_base, bool all_nodes, cudaStream_t st) {
        if (count == 0) return;
        const uint32_t R  = p.degree;
        const uint32_t MV = p.max_visited;
        vis_ids.ensure(sizeof(uint32_t) * count * MV);
        vis_d.ensure(sizeof(float) * count * MV);
        vis_n.ensure(sizeof(uint32_t) * count);

        vann::SearchArgs a{};
        a.store = vecs;
        a.vecs_f32 = vecs;
        a.deg = deg;
        a.adj = adj;
        a.adj_h = adj_h;
        a.R = R;
        a.tomb = tomb;
        a.queries = d_q;
        a.nq = count;
        a.D = p.dim;
        a.L = p.build_L;
        a.k = 0;
        a.entry = entry;
        a.max_hops = 1000000u;
        a.skip_mode = skip_mode;
        a.skip_base = skip_base;
        a.vis_ids = vis_ids.as<uint32_t>();
        a.vis_d = vis_d.as<float>();
        a.vis_n = vis_n.as<uint32_t>();
        a.max_visited = MV;
        a.order = search_order(d_q, count, st);
        a.counter = next_counter(st);
        a.status = status;
        // exact uint8 rows give the FP32 distances bit for bit from a quarter of the bytes
        int sstore = VANN_STORE_F32;
        if (u8_exact(st)) {
            a.store       = store[3];
            sstore        = VANN_STORE_U8;
            a.int_queries = 1;  // the batch's rows are rows of the exact copy
        }
        // the first large batch of each row format times the launch-bound variants
        // (the same search each time: the expansion lists do not depend on the variant)
        if (build_variant[sstore] < 0 && count >= 4096) {
            cudaEvent_t e0, e1;
            VCHECK(cudaEventCreate(&e0));
            VCHECK(cudaEventCreate(&e1));
            float best_ms = 1e30f;
            int   best    = 0;
            for (int v = 0; v < vann::search_variants(); ++v) {
                a.counter = next_counter(st);
                VCHECK(cudaEventRecord(e0, st));
                VCHECK(vann::launch_search(a, sstore, num_sms, st, v));
                VCHECK(cudaEventRecord(e1, st));
                VCHECK(cudaEventSynchronize(e1));
                float ms = 0.f;
                VCHECK(cudaEventElapsedTime(&ms, e0, e1));
                if (ms < best_ms) {
                    best_ms = ms;
                    best    = v;
                }
            }
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            build_variant[sstore] = best;
            a.counter = next_counter(st);
        }
        VCHECK(vann::launch_search(a, sstore, num_sms, st, std::max(build_variant[sstore], 0)));

        vann::PruneArgs pa{};
        pa.vecs = vecs;
        pa.D = p.dim;
        pa.deg = deg;
        pa.adj = adj;
        pa.adj_h = adj_h;
        pa.R = R;
        pa.alpha = p.alpha;
        pa.cap = MV;
        pa.node_ids = d_nodes;
        pa.n_nodes = count;
        pa.a_ids = vis_ids.as<uint32_t>();
        pa.a_d = vis_d.as<float>();
        pa.a_n = vis_n.as<uint32_t>();
        pa.a_stride = MV;
        pa.use_b = 1;
        pa.consistent = 0;
        pa.counter = next_counter(st);
        pa.status = status;
        run_prune(pa, st);

        // reverse edges, sorted by target with sources in batch order (stable)
        const uint64_t ne             = count * R;
        const bool     consistent_rev = consistent || all_nodes;
        e_keys.ensure(sizeof(uint32_t) * ne);
        e_vals.ensure(sizeof(uint32_t) * ne);
        e_keys2.ensure(sizeof(uint32_t) * ne);
        e_vals2.ensure(sizeof(uint32_t) * ne);
        const int end_bit = 32;  // padded slots carry UINT32_MAX keys
        vann::PruneArgs ra{};
        ra.vecs = vecs;
        ra.D = p.dim;
        ra.deg = deg;
        ra.adj = adj;
        ra.adj_h = adj_h;
        ra.R = R;
        ra.alpha = p.alpha;
        ra.cap = p.max_reverse;
        ra.csr_src = e_vals2.as<uint32_t>();
        ra.use_b = 1;
        ra.status = status;
        if (consistent_rev) {
            // Only the targets of new edges change: their ids and source runs come
            // from a run-length encoding of the sorted edge list, so this pass costs
            // O(batch * R), not O(index size).
            runs.ensure(3 * sizeof(uint32_t) * ne + 16);
            uint32_t* uniq   = runs.as<uint32_t>();
            uint32_t* runcnt = uniq + ne;
            uint32_t* runoff = runcnt + ne;
            uint32_t* nruns  = runoff + ne;
            VCHECK(vann::launch_edges(d_nodes, count, deg, adj, R, e_keys.as<uint32_t>(),
                                      e_vals.as<uint32_t>(), nullptr, st));
            size_t tmp_sort = 0, tmp_rle = 0, tmp_scan = 0;
            VCHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, e_keys.as<uint32_t>(),
                                                   e_keys2.as<uint32_t>(), e_vals.as<uint32_t>(),
                                                   e_vals2.as<uint32_t>(), (int)ne, 0, end_bit, st));
            VCHECK(cub::DeviceRunLengthEncode::Encode(nullptr, tmp_rle, e_keys2.as<uint32_t>(), uniq, runcnt,
                                                      nruns, (int)ne, st));
            VCHECK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, runcnt, runoff, (int)ne, st));
            cub_tmp.ensure(std::max(tmp_sort, std::max(tmp_rle, tmp_scan)));
            size_t t1 = cub_tmp.bytes, t2 = cub_tmp.bytes, t3 = cub_tmp.bytes;
            VCHECK(cub::DeviceRadixSort::SortPairs(cub_tmp.p, t1, e_keys.as<uint32_t>(),
                                                   e_keys2.as<uint32_t>(), e_vals.as<uint32_t>(),
                                                   e_vals2.as<uint32_t>(), (int)ne, 0, end_bit, st));
            VCHECK(cub::DeviceRunLengthEncode::Encode(cub_tmp.p, t2, e_keys2.as<uint32_t>(), uniq, runcnt, nruns,
                                                      (int)ne, st));
            // runs beyond the count hold stale values; their offsets are never read
            VCHECK(cub::DeviceScan::ExclusiveSum(cub_tmp.p, t3, runcnt, runoff, (int)ne, st));
            uint32_t hn = 0;
            VCHECK(cudaMemcpyAsync(&hn, nruns, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            VCHECK(cudaStreamSynchronize(st));
            ra.node_ids    = uniq;  // the run of padded slots (id UINT32_MAX) is skipped
            ra.n_nodes     = hn;
            ra.csr_off     = runoff;
            ra.csr_cnt     = runcnt;
            ra.csr_by_slot = 1;
            ra.skip_empty  = 0;
            ra.consistent  = 1;
        } else {
            // lists of unknown origin: the reference's literal pass over every node
            counts.ensure(sizeof(uint32_t) * (p.capacity + 1));
            offsets.ensure(sizeof(uint32_t) * (p.capacity + 1));
            VCHECK(cudaMemsetAsync(counts.p, 0, sizeof(uint32_t) * (size + 1), st));
            VCHECK(vann::launch_edges(d_nodes, count, deg, adj, R, e_keys.as<uint32_t>(),
                                      e_vals.as<uint32_t>(), counts.as<uint32_t>(), st));
            size_t tmp_sort = 0, tmp_scan = 0;
            VCHECK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_sort, e_keys.as<uint32_t>(),
                                                   e_keys2.as<uint32_t>(), e_vals.as<uint32_t>(),
                                                   e_vals2.as<uint32_t>(), (int)ne, 0, end_bit, st));
            VCHECK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, counts.as<uint32_t>(),
                                                 offsets.as<uint32_t>(), (int)(size + 1), st));
            cub_tmp.ensure(std::max(tmp_sort, tmp_scan));
            size_t t1 = cub_tmp.bytes, t2 = cub_tmp.bytes;
            VCHECK(cub::DeviceRadixSort::SortPairs(cub_tmp.p, t1, e_keys.as<uint32_t>(),
                                                   e_keys2.as<uint32_t>(), e_vals.as<uint32_t>(),
                                                   e_vals2.as<uint32_t>(), (int)ne, 0, end_bit, st));
            VCHECK(cub::DeviceScan::ExclusiveSum(cub_tmp.p, t2, counts.as<uint32_t>(),
                                                 offsets.as<uint32_t>(), (int)(size + 1), st));
            ra.node_ids   = nullptr;
            ra.n_nodes    = size;
            ra.csr_off    = offsets.as<uint32_t>();
            ra.csr_cnt    = counts.as<uint32_t>();
            ra.skip_empty = 0;
            ra.consistent = 0;
        }
        ra.counter = next_counter(st);
        run_prune(ra, st);
        consistent = true;
    }
};

namespace {

vann_status guard(const std::function<void()>& f) {
    try {
        f();
        return VANN_OK;
    } catch (const Fail& e) {
        return e.st;
    } catch (const std::bad_alloc&) {
        set_err("host allocation failed");
        return VANN_ERR_OOM;
    } catch (...) {
        set_err("unexpected exception");
        return VANN_ERR_INVALID;
    }
}

cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

extern "C" {

const char* vann_status_string(vann_status s) {
    switch (s) {
        case VANN_OK: return "ok";
        case VANN_ERR_INVALID: return "invalid argument";
        case VANN_ERR_CUDA: return "CUDA error";
        case VANN_ERR_CAPACITY: return "capacity exhausted";
        case VANN_ERR_IO: return "I/O error";
        case VANN_ERR_HOP_LIMIT: return "hop limit reached";
        case VANN_ERR_NOT_FOUND: return "not found";
        case VANN_ERR_TIMEOUT: return "timeout";
        case VANN_ERR_OOM: return "out of memory";
        case VANN_ERR_UNSUPPORTED: return "unsupported";
        case VANN_ERR_STATE: return "invalid state";
    }
    return "unknown";
}

const char* vann_last_error(void) { return g_last_error.c_str(); }
int         vann_abi_version(void) { return VANN_ABI_VERSION; }

vann_status vann_create(const vann_params* params, vann_index** out) {
    return guard([&] {
        VREQUIRE(params && out, VANN_ERR_INVALID, "null argument");
        const vann_params& p = *params;
        VREQUIRE(p.dim >= 4 && p.dim % 4 == 0 && p.dim <= 512, VANN_ERR_UNSUPPORTED,
                 "dim must be a multiple of 4 in [4, 512]");
        VREQUIRE(p.degree >= 1 && p.degree <= 128, VANN_ERR_UNSUPPORTED, "degree must be in [1, 128]");
        VREQUIRE(p.build_L >= 1 && p.build_L <= 1024, VANN_ERR_INVALID, "build_L must be in [1, 1024]");
        VREQUIRE(p.capacity >= 1 && p.capacity < 0x7fffffffull, VANN_ERR_INVALID,
                 "capacity must be in [1, 2^31-1)");
        VREQUIRE(p.max_visited >= 1 && p.max_visited <= 2048, VANN_ERR_INVALID,
                 "max_visited must be in [1, 2048]");
        VREQUIRE(p.max_reverse >= 1 && p.max_reverse <= 2048, VANN_ERR_INVALID,
                 "max_reverse must be in [1, 2048]");
        VREQUIRE(p.alpha >= 1.0f, VANN_ERR_INVALID, "alpha must be >= 1");
        VREQUIRE(!(p.stores & (1u << VANN_STORE_BF16)) || p.dim % 8 == 0, VANN_ERR_UNSUPPORTED,
                 "the bf16 copy needs dim to be a multiple of 8");
        VREQUIRE(!(p.stores & ((1u << VANN_STORE_FP8) | (1u << VANN_STORE_U8))) || p.dim % 16 == 0,
                 VANN_ERR_UNSUPPORTED, "one-byte copies need dim to be a multiple of 16");
        VREQUIRE(!(p.stores & (1u << VANN_STORE_PQ)) || p.dim % 128 == 0, VANN_ERR_UNSUPPORTED,
                 "the PQ copy needs dim to be a multiple of 128");
        auto* h = new vann_index();
        try {
            h->p = p;
            VCHECK(cudaGetDevice(&h->device));
            VCHECK(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
            const uint64_t C = p.capacity;
            h->alloc((void**)&h->vecs, sizeof(float) * C * p.dim);
            if (p.stores & (1u << VANN_STORE_BF16)) h->alloc(&h->store[1], 2ull * C * p.dim);
            if (p.stores & (1u << VANN_STORE_FP8)) {
                h->alloc(&h->store[2], 1ull * C * p.dim);
                h->alloc((void**)&h->fp8_scale, sizeof(float2) * C);
                h->alloc((void**)&h->fp8_center, sizeof(float) * p.dim);
            }
            if (p.stores & (1u << VANN_STORE_U8)) {
                h->alloc(&h->store[3], 1ull * C * p.dim);
                h->alloc((void**)&h->u8_lo, sizeof(float) * p.dim);
                h->alloc((void**)&h->u8_grid, sizeof(float) * 4);
            }
            if (p.stores & (1u << VANN_STORE_PQ)) {
                h->alloc(&h->store[4], 1ull * C * (p.dim / vann::kPqSub));
                h->alloc((void**)&h->pq_cb, sizeof(float) * (size_t)p.dim * vann::kPqK);
                h->alloc((void**)&h->pq_cnorm, sizeof(float) * (p.dim / vann::kPqSub));
            }
            h->store[0] = h->vecs;
            h->alloc((void**)&h->deg, sizeof(uint32_t) * C);
            h->alloc((void**)&h->adj, sizeof(uint32_t) * C * p.degree);
            h->alloc((void**)&h->adj_h, sizeof(uint32_t) * C * p.degree);
            h->alloc((void**)&h->tomb, sizeof(uint32_t) * h->tomb_words());
            h->alloc((void**)&h->counters, sizeof(uint32_t) * 32 * kCounterRing);
            h->alloc((void**)&h->status, sizeof(uint32_t) * 32);
            VCHECK(cudaMemset(h->deg, 0, sizeof(uint32_t) * C));
            VCHECK(cudaMemset(h->tomb, 0, sizeof(uint32_t) * h->tomb_words()));
            VCHECK(cudaMemset(h->status, 0, sizeof(uint32_t) * 32));
            VCHECK(cudaDeviceSynchronize());
        } catch (...) {
            h->store[0] = nullptr;
            delete h;
            throw;
        }
        *out = h;
    });
}

vann_status vann_destroy(vann_index* h) {
    return guard([&] {
        if (!h) return;
        cudaDeviceSynchronize();
        h->store[0] = nullptr;  // alias of vecs
        delete h;
    });
}

vann_status vann_get_info(const vann_index* h, vann_info* out) {
    return guard([&] {
        VREQUIRE(h && out, VANN_ERR_INVALID, "null argument");
        out->size = h->size;
        out->capacity = h->p.capacity;
        out->live = h->size - h->n_deleted - h->free_ids.size();
        out->free_ids = h->free_ids.size();
        out->entry = h->entry;
        out->dim = h->p.dim;
        out->degree = h->p.degree;
        out->consistent = h->consistent ? 1u : 0u;
        out->device_bytes = h->held;
        unsigned long long pr[2] = {0, 0};
        VCHECK(cudaMemcpy(pr, h->status + vann::kWordPruned, sizeof(pr), cudaMemcpyDeviceToHost));
        out->pruned_tc   = pr[0];
        out->pruned_cuda = pr[1];
        out->staged      = h->stage_n;
    });
}

vann_status vann_set_graph(vann_index* h, const float* h_vecs, const uint32_t* h_deg,
                           const uint32_t* h_adj, uint64_t n, uint32_t entry, uint32_t consistent) {
    return guard([&] {
        VREQUIRE(h && h_vecs && h_deg && h_adj, VANN_ERR_INVALID, "null argument");
        VREQUIRE(n <= h->p.capacity, VANN_ERR_CAPACITY, "n exceeds capacity");
        VREQUIRE(n == 0 || entry < n, VANN_ERR_INVALID, "entry must be < n");
        const uint32_t R = h->p.degree;
        for (uint64_t i = 0; i < n; ++i) {
            VREQUIRE(h_deg[i] <= R, VANN_ERR_INVALID, "degree exceeds R");
            for (uint32_t j = 0; j < h_deg[i]; ++j)
                VREQUIRE(h_adj[i * R + j] < n, VANN_ERR_INVALID, "neighbour id out of range");
        }
        VCHECK(cudaMemcpy(h->vecs, h_vecs, sizeof(float) * n * h->p.dim, cudaMemcpyHostToDevice));
        VCHECK(cudaMemcpy(h->deg, h_deg, sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
        VCHECK(cudaMemcpy(h->adj, h_adj, sizeof(uint32_t) * n * R, cudaMemcpyHostToDevice));
        VCHECK(vann::launch_hash_rows(h->adj, h->adj_h, n, R, 0));
        VCHECK(cudaMemset(h->tomb, 0, sizeof(uint32_t) * h->tomb_words()));
        h->convert_rows(0, n, 0);
        VCHECK(cudaDeviceSynchronize());
        h->size = n;
        h->n_deleted = 0;
        h->free_ids.clear();
        h->entry = entry;
        h->consistent = consistent != 0;
    });
}

vann_status vann_get_graph(vann_index* h, float* h_vecs, uint32_t* h_deg, uint32_t* h_adj) {
    return guard([&] {
        VREQUIRE(h, VANN_ERR_INVALID, "null argument");
        VCHECK(cudaDeviceSynchronize());
        if (h_vecs)
            VCHECK(cudaMemcpy(h_vecs, h->vecs, sizeof(float) * h->size * h->p.dim, cudaMemcpyDeviceToHost));
        if (h_deg) VCHECK(cudaMemcpy(h_deg, h->deg, sizeof(uint32_t) * h->size, cudaMemcpyDeviceToHost));
        if (h_adj)
            VCHECK(cudaMemcpy(h_adj, h->adj, sizeof(uint32_t) * h->size * h->p.degree,
                              cudaMemcpyDeviceToHost));
    });
}

vann_status vann_load_graph(vann_index* h, const char* path, uint64_t n, uint32_t entry) {
    return guard([&] {
        VREQUIRE(h && path, VANN_ERR_INVALID, "null argument");
        const uint32_t D = h->p.dim, R = h->p.degree;
        const size_t   rec = 4ull * D + 4 + 4ull * R;
        FILE*          f   = fopen(path, "rb");
        VREQUIRE(f, VANN_ERR_IO, std::string("cannot open ") + path);
        std::vector<unsigned char> buf(rec * n);
        size_t got = fread(buf.data(), rec, n, f);
        fclose(f);
        VREQUIRE(got == n, VANN_ERR_IO, "short read");
        std::vector<float>    v(n * D);
        std::vector<uint32_t> d(n), a(n * R);
        for (uint64_t i = 0; i < n; ++i) {
            const unsigned char* r = buf.data() + i * rec;
            memcpy(&v[i * D], r, 4ull * D);
            memcpy(&d[i], r + 4ull * D, 4);
            memcpy(&a[i * R], r + 4ull * D + 4, 4ull * R);
            // unused slots of the file may hold anything; keep them in range
            for (uint32_t j = d[i] < R ? d[i] : R; j < R; ++j) a[i * R + j] = 0;
        }
        vann_status s = vann_set_graph(h, v.data(), d.data(), a.data(), n, entry, 0);
        VREQUIRE(s == VANN_OK, s, g_last_error);
    });
}

vann_status vann_save_graph(vann_index* h, const char* path) {
    return guard([&] {
        VREQUIRE(h && path, VANN_ERR_INVALID, "null argument");
        const uint32_t D = h->p.dim, R = h->p.degree;
        const uint64_t n = h->size;
        std::vector<float>    v(n * D);
        std::vector<uint32_t> d(n), a(n * R);
        vann_status           s = vann_get_graph(h, v.data(), d.data(), a.data());
        VREQUIRE(s == VANN_OK, s, g_last_error);
        const size_t               rec = 4ull * D + 4 + 4ull * R;
        std::vector<unsigned char> buf(rec * n);
        for (uint64_t i = 0; i < n; ++i) {
            unsigned char* r = buf.data() + i * rec;
            memcpy(r, &v[i * D], 4ull * D);
            memcpy(r + 4ull * D, &d[i], 4);
            memset(r + 4ull * D + 4, 0, 4ull * R);
            memcpy(r + 4ull * D + 4, &a[i * R], 4ull * d[i]);
        }
        FILE* f = fopen(path, "wb");
        VREQUIRE(f, VANN_ERR_IO, std::string("cannot open ") + path);
        size_t put = fwrite(buf.data(), rec, n, f);
        fclose(f);
        VREQUIRE(put == n, VANN_ERR_IO, "short write");
    });
}

}  // extern "C"

namespace vann {
vann_status write_bang(std::vector<unsigned char>& records, uint64_t n, uint32_t dim, uint32_t degree,
                       uint32_t medoid, const char* out_prefix);
}

namespace {

// the index's graph as the reference's records (unused slots zero)
std::vector<unsigned char> graph_records(vann_index* h) {
    const uint32_t        D = h->p.dim, R = h->p.degree;
    const uint64_t        n = h->size;
    std::vector<float>    v(n * D);
    std::vector<uint32_t> d(n), a(n * R);
    vann_status           s = vann_get_graph(h, v.data(), d.data(), a.data());
    VREQUIRE(s == VANN_OK, s, g_last_error);
    const size_t               rec = 4ull * D + 4 + 4ull * R;
    std::vector<unsigned char> buf(rec * n);
    for (uint64_t i = 0; i < n; ++i) {
        unsigned char* r = buf.data() + i * rec;
        memcpy(r, &v[i * D], 4ull * D);
        memcpy(r + 4ull * D, &d[i], 4);
        memset(r + 4ull * D + 4, 0, 4ull * R);
        memcpy(r + 4ull * D + 4, &a[i * R], 4ull * d[i]);
    }
    return buf;
}

struct IndexFileHeader {
    char     magic[8];
    uint32_t version, dim, degree, consistent;
    uint64_t size, deleted, n_free;
    uint32_t entry, reserved;
};
static_assert(sizeof(IndexFileHeader) == 56, "file header layout");

}  // namespace

extern "C" {

vann_status vann_save_graph_bang(vann_index* h, const char* out_prefix) {
    vann_status written = VANN_OK;
    vann_status s       = guard([&] {
        VREQUIRE(h && out_prefix, VANN_ERR_INVALID, "null argument");
        std::vector<unsigned char> buf = graph_records(h);
        written = vann::write_bang(buf, h->size, h->p.dim, h->p.degree, h->entry, out_prefix);
    });
    return s != VANN_OK ? s : written;
}

vann_status vann_save_index(vann_index* h, const char* path) {
    return guard([&] {
        VREQUIRE(h && path, VANN_ERR_INVALID, "null argument");
        const uint32_t D = h->p.dim, R = h->p.degree;
        const uint64_t n = h->size;
        std::vector<float>    v(n * D);
        std::vector<uint32_t> d(n), a(n * R), tomb((n + 31) / 32);
        vann_status           s = vann_get_graph(h, v.data(), d.data(), a.data());
        VREQUIRE(s == VANN_OK, s, g_last_error);
        if (n) VCHECK(cudaMemcpy(tomb.data(), h->tomb, 4 * tomb.size(), cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < n; ++i)  // unused slots are not part of the state
            for (uint32_t j = d[i]; j < R; ++j) a[i * R + j] = 0;
        IndexFileHeader hd{};
        memcpy(hd.magic, "VANNIDX", 8);
        hd.version    = 1;
        hd.dim        = D;
        hd.degree     = R;
        hd.consistent = h->consistent ? 1u : 0u;
        hd.size       = n;
        hd.deleted    = h->n_deleted;
        hd.n_free     = h->free_ids.size();
        hd.entry      = h->entry;
        FILE* f = fopen(path, "wb");
        VREQUIRE(f, VANN_ERR_IO, std::string("cannot open ") + path);
        bool ok = fwrite(&hd, sizeof(hd), 1, f) == 1;
        ok      = ok && fwrite(v.data(), 4, v.size(), f) == v.size();
        ok      = ok && fwrite(d.data(), 4, d.size(), f) == d.size();
        ok      = ok && fwrite(a.data(), 4, a.size(), f) == a.size();
        ok      = ok && fwrite(tomb.data(), 4, tomb.size(), f) == tomb.size();
        ok      = ok && fwrite(h->free_ids.data(), 4, h->free_ids.size(), f) == h->free_ids.size();
        ok      = fclose(f) == 0 && ok;
        VREQUIRE(ok, VANN_ERR_IO, "short write");
    });
}

vann_status vann_load_index(vann_index* h, const char* path) {
    return guard([&] {
        VREQUIRE(h && path, VANN_ERR_INVALID, "null argument");
        FILE* f = fopen(path, "rb");
        VREQUIRE(f, VANN_ERR_IO, std::string("cannot open ") + path);
        IndexFileHeader hd{};
        bool            ok = fread(&hd, sizeof(hd), 1, f) == 1;
        if (!ok || memcmp(hd.magic, "VANNIDX", 8) != 0 || hd.version != 1) {
            fclose(f);
            VREQUIRE(false, VANN_ERR_IO, "not a version-1 index file");
        }
        if (hd.dim != h->p.dim || hd.degree != h->p.degree || hd.size > h->p.capacity ||
            hd.n_free > hd.size || hd.deleted > hd.size) {
            fclose(f);
            VREQUIRE(false, VANN_ERR_INVALID, "file dim / degree / size do not fit this index");
        }
        const uint64_t        n = hd.size, D = hd.dim, R = hd.degree;
        std::vector<float>    v(n * D);
        std::vector<uint32_t> d(n), a(n * R), tomb((n + 31) / 32), fr(hd.n_free);
        ok = fread(v.data(), 4, v.size(), f) == v.size();
        ok = ok && fread(d.data(), 4, d.size(), f) == d.size();
        ok = ok && fread(a.data(), 4, a.size(), f) == a.size();
        ok = ok && fread(tomb.data(), 4, tomb.size(), f) == tomb.size();
        ok = ok && fread(fr.data(), 4, fr.size(), f) == fr.size();
        fclose(f);
        VREQUIRE(ok, VANN_ERR_IO, "short read");
        for (uint32_t x : fr) VREQUIRE(x < n, VANN_ERR_INVALID, "free id out of range");
        vann_status s = vann_set_graph(h, v.data(), d.data(), a.data(), n, hd.entry, hd.consistent);
        VREQUIRE(s == VANN_OK, s, g_last_error);
        if (n) VCHECK(cudaMemcpy(h->tomb, tomb.data(), 4 * tomb.size(), cudaMemcpyHostToDevice));
        h->n_deleted = hd.deleted;
        h->free_ids.assign(fr.begin(), fr.end());
    });
}

vann_status vann_build(vann_index* h, const float* d_vecs, uint64_t n, uint64_t batch, uint64_t seed,
                       uint32_t entry, void* stream) {
    return guard([&] {
        VREQUIRE(h && (d_vecs || n == 0), VANN_ERR_INVALID, "null argument");
        VREQUIRE(n <= h->p.capacity, VANN_ERR_CAPACITY, "n exceeds capacity");
        cudaStream_t   st = S(stream);
        const uint32_t D = h->p.dim, R = h->p.degree;
        h->size = 0;
        h->n_deleted = 0;
        h->free_ids.clear();
        h->consistent = false;
        if (n == 0) return;
        VCHECK(cudaMemcpyAsync(h->vecs, d_vecs, sizeof(float) * n * D, cudaMemcpyDeviceToDevice, st));
        VCHECK(cudaMemsetAsync(h->tomb, 0, sizeof(uint32_t) * h->tomb_words(), st));
        VCHECK(cudaMemsetAsync(h->deg, 0, sizeof(uint32_t) * n, st));
        h->convert_rows(0, n, st);
        const uint64_t first = (batch == 0 || batch >= n) ? n : batch;
        VCHECK(vann::launch_random_graph(h->deg, h->adj, h->adj_h, 0, first, R, seed, st));
        h->size  = first;
        h->entry = entry != vann::kNone ? entry : h->medoid(first, st);
        VREQUIRE(h->entry < first, VANN_ERR_INVALID, "entry must be inside the first batch");
        const bool parity = (h->p.flags & VANN_QUIRK_SKIP_BATCH_INDEX) != 0;
        const uint64_t step = first;
        h->nodes.ensure(sizeof(uint32_t) * (batch == 0 || batch >= n ? n : batch));
        VCHECK(vann::launch_iota(h->nodes.as<uint32_t>(), first, 0, st));
        h->vamana_batch(h->nodes.as<uint32_t>(), first, h->vecs, parity ? 1u : 2u, 0u, true, st);
        for (uint64_t s = first; s < n; s += step) {
            uint64_t c = std::min(step, n - s);
            h->size    = s + c;
            VCHECK(vann::launch_iota(h->nodes.as<uint32_t>(), c, (uint32_t)s, st));
            h->vamana_batch(h->nodes.as<uint32_t>(), c, h->vecs + s * D, parity ? 1u : 0u, 0u, false, st);
        }
        VCHECK(cudaStreamSynchronize(st));
        VCHECK(cudaGetLastError());
        h->check_device_status();
    });
}

vann_status vann_build_loaded(vann_index* h, void* stream) {
    return guard([&] {
        VREQUIRE(h, VANN_ERR_INVALID, "null argument");
        VREQUIRE(h->size > 0 && h->entry < h->size, VANN_ERR_STATE, "load or set a graph first");
        cudaStream_t st = S(stream);
        const bool   parity = (h->p.flags & VANN_QUIRK_SKIP_BATCH_INDEX) != 0;
        h->consistent = false;
        h->nodes.ensure(sizeof(uint32_t) * h->size);
        VCHECK(vann::launch_iota(h->nodes.as<uint32_t>(), h->size, 0, st));
        h->vamana_batch(h->nodes.as<uint32_t>(), h->size, h->vecs, parity ? 1u : 2u, 0u, true, st);
        VCHECK(cudaStreamSynchronize(st));
        h->check_device_status();
    });
}

vann_status vann_search_stats(vann_index* h, const float* d_queries, uint64_t nq,
                              const vann_search_params* sp, uint32_t* d_ids, float* d_dists,
                              uint32_t* d_hops, uint32_t* d_evals, uint32_t* d_adjw, void* stream) {
    return guard([&] {
        VREQUIRE(h && sp && (nq == 0 || (d_queries && d_ids && d_dists)), VANN_ERR_INVALID,
                 "null argument");
        VREQUIRE(sp->k >= 1 && sp->L >= sp->k && sp->L <= 1024, VANN_ERR_INVALID,
                 "need 1 <= k <= L <= 1024");
        VREQUIRE(sp->store < 5 && h->store[sp->store] != nullptr, VANN_ERR_UNSUPPORTED,
                 "requested store was not enabled at create");
        VREQUIRE(sp->beam <= 2, VANN_ERR_INVALID, "beam must be 0, 1 or 2");
        VREQUIRE(sp->beam < 2 || (sp->L <= 64 && h->p.dim <= 128 && h->p.degree <= 64), VANN_ERR_UNSUPPORTED,
                 "beam 2 needs L <= 64, dim <= 128 and degree <= 64");
        VREQUIRE(h->size > 0 && h->entry < h->size, VANN_ERR_STATE, "index is empty");
        if (nq == 0) return;
        vann::SearchArgs a{};
        a.beam  = vann_index::beam_of(*sp);
        a.store = h->store[sp->store];
        a.scale = h->fp8_scale;
        a.center = sp->store == VANN_STORE_FP8 ? h->fp8_center : nullptr;
        a.pq_cb = h->pq_cb;
        a.pq_cnorm = h->pq_cnorm;
        a.vecs_f32 = h->vecs;
        a.deg = h->deg;
        a.adj = h->adj;
        a.adj_h = h->adj_h;
        a.R = h->p.degree;
        a.tomb = h->n_deleted || !h->free_ids.empty() ? h->tomb : nullptr;
        a.queries = d_queries;
        a.nq = nq;
        a.D = h->p.dim;
        a.L = sp->L;
        a.k = sp->k;
        a.entry = h->entry;
        a.max_hops = sp->max_hops ? sp->max_hops : 1000000u;
        a.skip_mode = (sp->flags & VANN_QUIRK_SKIP_BATCH_INDEX) ? 1u : 0u;
        a.rerank = sp->rerank ? 1 : 0;
        a.out_ids = d_ids;
        a.out_d = d_dists;
        a.hops_out = d_hops;
        a.evals_out = d_evals;
        a.adjw_out = d_adjw;
        a.Lq = h->pending_Lq;
        a.kq = h->pending_kq;
        // a search over the uint8 copy on a fitted grid needs a per-stream workspace (the
        // queries on the grid, and with rerank the candidate lists): sized here, before
        // anything is queued, and never allocated while the stream is being captured
        DevBuf* grid_ws = nullptr;
        if (sp->store == VANN_STORE_U8 && h->u8_affine) {
            const size_t need = sizeof(float) * nq * h->p.dim +
                                (sp->rerank ? (sizeof(uint32_t) + sizeof(float)) * nq * sp->L : 0);
            grid_ws = &h->grid_ws[S(stream)];
            if (grid_ws->bytes < need) {
                cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                VCHECK(cudaStreamIsCapturing(S(stream), &cs));
                VREQUIRE(cs == cudaStreamCaptureStatusNone, VANN_ERR_STATE,
                         "a search over the fitted uint8 grid needs its workspace before capture: run one "
                         "search of this size on the stream first");
                if (grid_ws->p) {  // a captured search may hold the old one: keep it until destroy
                    h->ord_retired.push_back(grid_ws->p);
                    grid_ws->p     = nullptr;
                    grid_ws->bytes = 0;
                }
                grid_ws->ensure(need);
            }
        }
        // the order kernel zeroes the counter, else a memset does
        a.counter  = h->next_counter(S(stream), false);
        bool chain = false;
        a.order    = h->search_order(d_queries, nq, S(stream), a.counter, &chain);
        if (a.order == nullptr) VCHECK(cudaMemsetAsync(a.counter, 0, sizeof(uint32_t), S(stream)));
        a.pdl = chain ? 1 : 0;
        a.status = h->status;
        if (grid_ws != nullptr) {
            // uint8 copy on a fitted grid: the queries rounded onto the grid, the search on
            // code distances, then the exact FP32 rerank of each list, or the distances
            // scaled back by s^2 (the queries' order above comes from the FP32 queries)
            cudaStream_t   st   = S(stream);
            const uint32_t L    = sp->L;
            const size_t   qb   = sizeof(float) * nq * h->p.dim;
            DevBuf&        ws   = *grid_ws;
            float*         qg   = ws.as<float>();
            VCHECK(vann::launch_grid_queries(d_queries, nq, h->p.dim, h->u8_lo, h->u8_inv, qg, st));
            a.queries = qg;
            a.rerank  = 0;
            if (sp->rerank) {
                uint32_t* cand = reinterpret_cast<uint32_t*>(static_cast<char*>(ws.p) + qb);
                a.k       = L;
                a.kq      = nullptr;  // every list whole: the rerank applies k
                a.out_ids = cand;
                a.out_d   = reinterpret_cast<float*>(cand + nq * L);
                VCHECK(vann::launch_search(a, (int)sp->store, h->num_sms, st, h->variant_for(*sp)));
                VCHECK(vann::launch_rerank(h->vecs, d_queries, nq, h->p.dim, cand, L, h->pending_kq, sp->k, d_ids,
                                           d_dists, h->num_sms, st));
            } else {
                VCHECK(vann::launch_search(a, (int)sp->store, h->num_sms, st, h->variant_for(*sp)));
                VCHECK(vann::launch_scale(d_dists, nq * sp->k, h->u8_s * h->u8_s, st));
            }
            return;
        }
        VCHECK(vann::launch_search(a, (int)sp->store, h->num_sms, S(stream), h->variant_for(*sp)));
    });
}

int vann_search_variant_count(void) { return vann::search_variants(); }

vann_status vann_stage_insert(vann_index* h, const float* d_vecs, uint64_t n, void* stream) {
    return guard([&] {
        VREQUIRE(h && (d_vecs || n == 0), VANN_ERR_INVALID, "null argument");
        if (n == 0) return;
        cudaStream_t st  = S(stream);
        const size_t row = sizeof(float) * h->p.dim;
        if ((h->stage_n + n) * row > h->stage.bytes) {  // grow by 1.5x, keeping the rows
            const size_t nb = std::max((h->stage_n + n) * row, h->stage.bytes * 3 / 2);
            void*        np = nullptr;
            VCHECK(cudaMalloc(&np, nb));
            cudaError_t e = h->stage_n ? cudaMemcpyAsync(np, h->stage.p, h->stage_n * row,
                                                         cudaMemcpyDeviceToDevice, st)
                                       : cudaSuccess;
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                cudaFree(np);
                VCHECK(e);
            }
            h->stage.release();
            h->stage.p     = np;
            h->stage.bytes = nb;
        }
        VCHECK(cudaMemcpyAsync(static_cast<char*>(h->stage.p) + h->stage_n * row, d_vecs, n * row,
                               cudaMemcpyDeviceToDevice, st));
        VCHECK(cudaStreamSynchronize(st));
        h->stage_n += n;
    });
}

vann_status vann_search_staged(vann_index* h, const float* d_queries, uint64_t nq, const vann_search_params* sp,
                               uint32_t* d_ids, float* d_dists, float* d_vecs_out, void* stream) {
    vann_status st_search = VANN_OK;
    vann_status s         = guard([&] {
        VREQUIRE(h && sp && (nq == 0 || (d_queries && d_ids && d_dists)), VANN_ERR_INVALID, "null argument");
        VREQUIRE(sp->L >= 1 && sp->L <= 1024, VANN_ERR_INVALID, "need 1 <= L <= 1024");
        if (nq == 0) return;
        cudaStream_t       st = S(stream);
        vann_search_params p  = *sp;
        p.k                   = p.L;  // the whole worklist, in its order
        h->s2_ids.ensure(sizeof(uint32_t) * nq * p.L);
        h->s2_d.ensure(sizeof(float) * nq * p.L);
        st_search = vann_search(h, d_queries, nq, &p, h->s2_ids.as<uint32_t>(), h->s2_d.as<float>(), stream);
        if (st_search != VANN_OK) return;
        vann::StagedArgs a{};
        a.queries   = d_queries;
        a.nq        = nq;
        a.vecs      = h->vecs;
        a.graph_ids = h->s2_ids.as<uint32_t>();
        a.L         = p.L;
        a.D         = h->p.dim;
        a.stage     = h->stage.as<float>();
        a.n_stage   = h->stage_n;
        a.out_ids   = d_ids;
        a.out_d     = d_dists;
        a.out_vecs  = d_vecs_out;
        VCHECK(vann::launch_staged_merge(a, h->num_sms, st));
    });
    return s != VANN_OK ? s : st_search;
}

vann_status vann_patch_graph(vann_index* h, uint32_t* d_ids_out, void* stream) {
    vann_status st_insert = VANN_OK;
    vann_status s         = guard([&] {
        VREQUIRE(h, VANN_ERR_INVALID, "null argument");
        if (h->stage_n == 0) return;
        st_insert = vann_insert(h, h->stage.as<float>(), h->stage_n, d_ids_out, stream);
        if (st_insert == VANN_OK) h->stage_n = 0;
    });
    return s != VANN_OK ? s : st_insert;
}

vann_status vann_autotune(vann_index* h, const float* d_queries, uint64_t nq, const vann_search_params* sp,
                          float* h_ms_out, void* stream) {
    return guard([&] {
        VREQUIRE(h && sp && d_queries && nq > 0, VANN_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        h->out_tmp.ensure((sizeof(uint32_t) + sizeof(float)) * nq * sp->k);
        uint32_t*   ids = h->out_tmp.as<uint32_t>();
        float*      dd  = reinterpret_cast<float*>(ids + nq * sp->k);
        cudaEvent_t e0, e1;
        VCHECK(cudaEventCreate(&e0));
        VCHECK(cudaEventCreate(&e1));
        const auto key = std::make_tuple(sp->store, sp->rerank ? 1u : 0u, vann_index::beam_of(*sp), sp->L);
        int   best = 0;
        float best_ms = 1e30f;
        for (int v = 0; v < vann::search_variants(); ++v) {
            h->tuned[key] = v;
            float ms_sum = 0.f;
            for (int rep = 0; rep < 4; ++rep) {
                VCHECK(cudaEventRecord(e0, st));
                vann_status s2 = vann_search(h, d_queries, nq, sp, ids, dd, stream);
                VREQUIRE(s2 == VANN_OK, s2, g_last_error);
                VCHECK(cudaEventRecord(e1, st));
                VCHECK(cudaEventSynchronize(e1));
                float ms = 0.f;
                VCHECK(cudaEventElapsedTime(&ms, e0, e1));
                if (rep > 0) ms_sum += ms;  // first run warms up
            }
            if (h_ms_out) h_ms_out[v] = ms_sum / 3.f;
            if (ms_sum < best_ms) {
                best_ms = ms_sum;
                best    = v;
            }
        }
        h->tuned[key] = best;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    });
}

vann_status vann_search(vann_index* h, const float* d_queries, uint64_t nq,
                        const vann_search_params* sp, uint32_t* d_ids, float* d_dists, void* stream) {
    return vann_search_stats(h, d_queries, nq, sp, d_ids, d_dists, nullptr, nullptr, nullptr, stream);
}

vann_status vann_search_uneven(vann_index* h, const float* d_queries, uint64_t nq, const vann_search_params* sp,
                               const uint32_t* d_L, const uint32_t* d_k, uint32_t* d_ids, float* d_dists,
                               void* stream) {
    h->pending_Lq = d_L;
    h->pending_kq = d_k;
    vann_status s = vann_search_stats(h, d_queries, nq, sp, d_ids, d_dists, nullptr, nullptr, nullptr, stream);
    h->pending_Lq = nullptr;
    h->pending_kq = nullptr;
    return s;
}

vann_status vann_sync(vann_index* h, void* stream) {
    vann_status result = VANN_OK;
    vann_status s = guard([&] {
        VREQUIRE(h, VANN_ERR_INVALID, "null argument");
        VCHECK(cudaStreamSynchronize(S(stream)));
        uint32_t w = 0;
        VCHECK(cudaMemcpy(&w, h->status, sizeof(w), cudaMemcpyDeviceToHost));
        VCHECK(cudaMemset(h->status, 0, sizeof(uint32_t)));
        if (w & vann::kStatusTimeout) {
            set_err("a bounded device wait gave up");
            result = VANN_ERR_TIMEOUT;
        } else if (w & vann::kStatusHopLimit) {
            set_err("a search stopped at its hop limit");
            result = VANN_ERR_HOP_LIMIT;
        }
    });
    return s != VANN_OK ? s : result;
}

vann_status vann_insert(vann_index* h, const float* d_vecs, uint64_t n, uint32_t* d_ids_out,
                        void* stream) {
    return guard([&] {
        VREQUIRE(h && (d_vecs || n == 0), VANN_ERR_INVALID, "null argument");
        VREQUIRE(h->size > 0, VANN_ERR_STATE, "build or load a graph first");
        if (n == 0) return;
        const uint64_t reuse = std::min<uint64_t>(n, h->free_ids.size());
        VREQUIRE(h->size + (n - reuse) <= h->p.capacity, VANN_ERR_CAPACITY, "capacity exhausted");
        cudaStream_t   st = S(stream);
        const uint32_t D  = h->p.dim;
        std::vector<uint32_t> ids(n);
        for (uint64_t i = 0; i < reuse; ++i) {
            ids[i] = h->free_ids.back();
            h->free_ids.pop_back();
        }
        for (uint64_t i = reuse; i < n; ++i) ids[i] = (uint32_t)(h->size + (i - reuse));
        h->nodes.ensure(sizeof(uint32_t) * n);
        VCHECK(cudaMemcpyAsync(h->nodes.p, ids.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st));
        scatter_rows_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(d_vecs, h->nodes.as<uint32_t>(), n,
                                                                     D, h->vecs, h->deg, h->tomb);
        VCHECK(cudaGetLastError());
        if (reuse == 0) {
            h->convert_rows(h->size, n, st);
        } else {
            h->u8_state = -1;
            for (int s = 1; s < 4; ++s)  // reused ids are scattered: convert by id list
                if (h->store[s])
                    VCHECK(vann::launch_convert_ids(h->vecs, h->nodes.as<uint32_t>(), n, h->store[s],
                                                    s == 2 ? h->fp8_scale : nullptr, h->copy_center(s), h->u8_inv,
                                                    D, s, h->u8_inexact(), st));
            if (h->store[4])
                VCHECK(vann::launch_pq_encode(h->vecs, 0, n, h->nodes.as<uint32_t>(), D, h->pq_cb,
                                              static_cast<uint8_t*>(h->store[4]), st));
        }
        h->size += n - reuse;
        const bool parity = (h->p.flags & VANN_QUIRK_SKIP_BATCH_INDEX) != 0;
        h->vamana_batch(h->nodes.as<uint32_t>(), n, d_vecs, parity ? 1u : 0u, 0u, false, st);
        if (d_ids_out)
            VCHECK(cudaMemcpyAsync(d_ids_out, h->nodes.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
        VCHECK(cudaStreamSynchronize(st));
        h->check_device_status();
    });
}

vann_status vann_delete(vann_index* h, const uint32_t* d_ids, uint64_t n, void* stream) {
    return guard([&] {
        VREQUIRE(h && (d_ids || n == 0), VANN_ERR_INVALID, "null argument");
        VCHECK(vann::launch_set_bits(h->tomb, d_ids, n, h->size, S(stream)));
        h->n_deleted += n;  // upper bound; recounted at consolidate
    });
}

vann_status vann_delete_by_vector(vann_index* h, const float* d_vecs, uint64_t n, int32_t* d_ids_out,
                                  void* stream) {
    return guard([&] {
        VREQUIRE(h && (d_vecs || n == 0), VANN_ERR_INVALID, "null argument");
        if (n == 0) return;
        cudaStream_t st = S(stream);
        h->out_tmp.ensure(sizeof(int32_t) * n);
        int32_t* res = d_ids_out ? d_ids_out : h->out_tmp.as<int32_t>();
        VCHECK(vann::launch_find_vectors(h->vecs, h->size, h->p.dim, d_vecs, n, h->tomb, res, st));
        std::vector<int32_t> hr(n);
        VCHECK(cudaMemcpyAsync(hr.data(), res, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
        VCHECK(cudaStreamSynchronize(st));
        std::vector<uint32_t> found;
        for (int32_t v : hr)
            if (v >= 0) found.push_back((uint32_t)v);
        if (!found.empty()) {
            h->nodes.ensure(sizeof(uint32_t) * found.size());
            VCHECK(cudaMemcpyAsync(h->nodes.p, found.data(), sizeof(uint32_t) * found.size(),
                                   cudaMemcpyHostToDevice, st));
            VCHECK(vann::launch_set_bits(h->tomb, h->nodes.as<uint32_t>(), found.size(), h->size, st));
            h->n_deleted += found.size();
            VCHECK(cudaStreamSynchronize(st));
        }
        VREQUIRE(found.size() == n, VANN_ERR_NOT_FOUND, "some vectors were not found");
    });
}

vann_status vann_consolidate(vann_index* h, void* stream) {
    return guard([&] {
        VREQUIRE(h, VANN_ERR_INVALID, "null argument");
        cudaStream_t   st = S(stream);
        const uint32_t R  = h->p.degree;
        // which ids are deleted and not yet free
        std::vector<uint32_t> tomb(h->tomb_words());
        VCHECK(cudaMemcpyAsync(tomb.data(), h->tomb, sizeof(uint32_t) * tomb.size(),
                               cudaMemcpyDeviceToHost, st));
        VCHECK(cudaStreamSynchronize(st));
        std::vector<char> is_free(h->size, 0);
        for (uint32_t f : h->free_ids) is_free[f] = 1;
        std::vector<uint32_t> dead;
        for (uint64_t i = 0; i < h->size; ++i)
            if (((tomb[i >> 5] >> (i & 31)) & 1u) && !is_free[i]) dead.push_back((uint32_t)i);
        if (dead.empty()) {
            h->n_deleted = 0;
            return;
        }
        const uint32_t cap = std::min<uint32_t>(2048u, std::max<uint32_t>(h->p.max_visited, 2 * R));
        // Nodes go in ranges whose candidate lists fit a fixed workspace (cap words per
        // node).  A node's candidates come from its own list and from deleted nodes'
        // lists, which no prune of this call changes, so the ranges give the same
        // graph as one pass over every node.
        constexpr uint64_t kCandBudget = uint64_t(512) << 20;
        const uint64_t     span = std::max<uint64_t>(1024, kCandBudget / (sizeof(uint32_t) * cap));
        const uint64_t     rng  = std::min<uint64_t>(h->size, span);
        h->nodes.ensure(sizeof(uint32_t) * rng);
        h->list_n.ensure(sizeof(uint32_t) * 4);
        h->cand.ensure(sizeof(uint32_t) * rng * cap);
        h->cand_n.ensure(sizeof(uint32_t) * rng);
        for (uint64_t lo = 0; lo < h->size; lo += rng) {
            const uint64_t cnt = std::min<uint64_t>(rng, h->size - lo);
            VCHECK(cudaMemsetAsync(h->list_n.p, 0, sizeof(uint32_t), st));
            VCHECK(vann::launch_consolidate_candidates(h->deg, h->adj, R, h->tomb, lo, cnt,
                                                       h->nodes.as<uint32_t>(), h->list_n.as<uint32_t>(),
                                                       h->cand.as<uint32_t>(), h->cand_n.as<uint32_t>(), cap,
                                                       h->num_sms, st));
            uint32_t nlist = 0;
            VCHECK(cudaMemcpyAsync(&nlist, h->list_n.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            VCHECK(cudaStreamSynchronize(st));
            if (nlist == 0) continue;
            vann::PruneArgs pa{};
            pa.vecs = h->vecs;
            pa.D = h->p.dim;
            pa.deg = h->deg;
            pa.adj = h->adj;
            pa.adj_h = h->adj_h;
            pa.R = R;
            pa.alpha = h->p.alpha;
            pa.cap = cap;
            pa.node_ids = h->nodes.as<uint32_t>();
            pa.n_nodes = nlist;
            pa.a_ids = h->cand.as<uint32_t>();
            pa.a_d = nullptr;  // computed by the prune
            pa.a_n = h->cand_n.as<uint32_t>();
            pa.a_stride = cap;
            pa.use_b = 0;
            pa.consistent = 0;
            pa.counter = h->next_counter(st);
            pa.status = h->status;
            h->run_prune(pa, st);
        }
        // free the deleted ids (tombstone stays set until an insert reuses the id)
        h->nodes.ensure(sizeof(uint32_t) * dead.size());
        VCHECK(cudaMemcpyAsync(h->nodes.p, dead.data(), sizeof(uint32_t) * dead.size(),
                               cudaMemcpyHostToDevice, st));
        clear_deg_kernel<<<(unsigned)((dead.size() + 255) / 256), 256, 0, st>>>(
            h->nodes.as<uint32_t>(), dead.size(), h->deg);
        VCHECK(cudaGetLastError());
        // a deleted entry point moves to the live node nearest to its vector,
        // found by a search that starts from the first live id
        if ((tomb[h->entry >> 5] >> (h->entry & 31)) & 1u) {
            uint32_t start = vann::kNone;
            for (uint64_t i = 0; i < h->size && start == vann::kNone; ++i)
                if (!((tomb[i >> 5] >> (i & 31)) & 1u)) start = (uint32_t)i;
            VREQUIRE(start != vann::kNone, VANN_ERR_STATE, "no live node left");
            h->out_tmp.ensure(sizeof(uint32_t) * 64 + sizeof(float) * h->p.dim);
            uint32_t* oi = h->out_tmp.as<uint32_t>();
            float*    od = reinterpret_cast<float*>(oi + 32);
            float*    qv = reinterpret_cast<float*>(oi + 64);
            VCHECK(cudaMemcpyAsync(qv, h->vecs + (uint64_t)h->entry * h->p.dim,
                                   sizeof(float) * h->p.dim, cudaMemcpyDeviceToDevice, st));
            vann::SearchArgs a{};
            a.store = h->vecs;
            a.vecs_f32 = h->vecs;
            a.deg = h->deg;
            a.adj = h->adj;
            a.adj_h = h->adj_h;
            a.R = R;
            a.tomb = h->tomb;
            a.queries = qv;
            a.nq = 1;
            a.D = h->p.dim;
            a.L = 32;
            a.k = 32;
            a.entry = start;
            a.max_hops = 1000000u;
            a.out_ids = oi;
            a.out_d = od;
            a.counter = h->next_counter(st);
            a.status = h->status;
            VCHECK(vann::launch_search(a, 0, h->num_sms, st));
            std::vector<uint32_t> res(32);
            VCHECK(cudaMemcpyAsync(res.data(), oi, sizeof(uint32_t) * 32, cudaMemcpyDeviceToHost, st));
            VCHECK(cudaStreamSynchronize(st));
            uint32_t ne = start;
            for (uint32_t r : res)
                if (r != vann::kNone && !((tomb[r >> 5] >> (r & 31)) & 1u)) {
                    ne = r;
                    break;
                }
            h->entry = ne;
        }
        for (uint32_t d : dead) h->free_ids.push_back(d);
        h->n_deleted = 0;
        VCHECK(cudaStreamSynchronize(st));
        h->check_device_status();
    });
}

}  // extern "C"

// vann.hpp -- header-only C++ mirror of the reference's index class over the C ABI.
//
// Drop-in for callers of the reference's `template <typename T> class Vamana`
// (vamana/include/vamana.cuh:36-146): same member names and argument meaning.
//   Vamana(graph_path, ...)    initGraph + runVamana (vamana_impl.cuh:10-20, 289-360)
//   insertPoints(d_vecs, n)    append to the insert list, outside the graph (vamana_impl.cuh:22-33)
//   deletePoints(d_vecs, n)    lazy delete by exact vector match (vamana_impl.cuh:35-53)
//   searchPoints(d_q, n)       device n x L worklist ids, caller cudaFree()s (vamana_impl.cuh:55-96)
//   searchPoints2(d_q, n)      graph results merged with the insert list; device n x L x D
//                              rows, caller cudaFree()s (vamana_impl.cuh:98-180)
//   patchGraph()               insert the insert list, consolidate deletes (vamana_impl.cuh:182-265)
//   saveGraph(path)            772-byte records at D=128, R=64 (vamana.cu:1346-1362)
// Error behaviour: the reference's gpuErrchk prints and exit()s (utils.cuh:68-78);
// this mirror throws vann::Error carrying the status and message instead.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "vann.h"

namespace vann {

struct Error : std::runtime_error {
    vann_status status;
    Error(vann_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(vann_status s) {
    if (s != VANN_OK) throw Error(s, std::string(vann_status_string(s)) + ": " + vann_last_error());
}

struct VamanaParams {
    uint32_t dim = 128, R = 64, L = 199;   // reference constants.cuh:7-10
    float    alpha = 1.5f;                 // vamana_impl.cuh:297
    uint32_t max_visited = 600, max_reverse = 500;
    bool     reference_quirks = true;      // batch-index skip, search.cuh:126
    double   capacity_factor = 1.3;        // utils.cuh:120
    uint64_t seed = 0;
};

template <typename T = float>
class Vamana {
    static_assert(sizeof(T) == 4, "the C ABI takes FP32 vectors");

   public:
    // initGraph(path) + runVamana: read n records (vectors + start graph) and
    // build over them with the reference's single-batch build.
    Vamana(const std::string& graph_path, uint64_t n, uint32_t medoid, const VamanaParams& p = {})
        : p_(p) {
        create(n);
        check(vann_load_graph(h_, graph_path.c_str(), n, medoid));
        check(vann_build_loaded(h_, nullptr));  // the file's adjacency is the start graph
    }
    // Build over n device vectors (seeded random start graph, medoid entry).
    Vamana(const T* d_vecs, uint64_t n, const VamanaParams& p = {}) : p_(p) {
        create(n);
        check(vann_build(h_, d_vecs, n, 0, p_.seed, 0xFFFFFFFFu, nullptr));
    }
    ~Vamana() {
        if (h_) vann_destroy(h_);
    }
    Vamana(const Vamana&) = delete;
    Vamana& operator=(const Vamana&) = delete;

    void insertPoints(T* d_query_vecs, size_t num) { check(vann_stage_insert(h_, d_query_vecs, num, nullptr)); }

    void deletePoints(T* d_query_vecs, size_t num) {
        if (num == 0) return;
        vann_status s = vann_delete_by_vector(h_, d_query_vecs, num, nullptr, nullptr);
        if (s != VANN_ERR_NOT_FOUND) check(s);  // the reference ignores vectors it cannot find
    }

    // n x L ids on the device (the reference returns its worklist); free with cudaFree.
    [[nodiscard]] uint32_t* searchPoints(T* d_query_vecs, size_t num) {
        uint32_t* ids = nullptr;
        float*    d   = nullptr;
        if (cudaMalloc(&ids, sizeof(uint32_t) * num * p_.L) != cudaSuccess ||
            cudaMalloc(&d, sizeof(float) * num * p_.L) != cudaSuccess)
            throw Error(VANN_ERR_OOM, "cudaMalloc");
        vann_search_params sp{p_.L, p_.L, VANN_STORE_F32, 0,
                              p_.reference_quirks ? VANN_QUIRK_SKIP_BATCH_INDEX : 0u, 0};
        vann_status s = vann_search(h_, d_query_vecs, num, &sp, ids, d, nullptr);
        cudaFree(d);
        check(s);
        check(vann_sync(h_, nullptr));
        return ids;
    }

    // n x L x D rows on the device (the reference's searchPoints2 result); free with cudaFree.
    [[nodiscard]] T* searchPoints2(T* d_query_vecs, size_t num) {
        uint32_t* ids  = nullptr;
        float*    d    = nullptr;
        T*        rows = nullptr;
        if (cudaMalloc(&ids, sizeof(uint32_t) * num * p_.L) != cudaSuccess ||
            cudaMalloc(&d, sizeof(float) * num * p_.L) != cudaSuccess ||
            cudaMalloc(&rows, sizeof(T) * num * p_.L * p_.dim) != cudaSuccess) {
            cudaFree(ids);
            cudaFree(d);
            throw Error(VANN_ERR_OOM, "cudaMalloc");
        }
        vann_search_params sp{p_.L, p_.L, VANN_STORE_F32, 0,
                              p_.reference_quirks ? VANN_QUIRK_SKIP_BATCH_INDEX : 0u, 0};
        vann_status s = vann_search_staged(h_, d_query_vecs, num, &sp, ids, d, rows, nullptr);
        if (s == VANN_OK) s = vann_sync(h_, nullptr);
        cudaFree(ids);
        cudaFree(d);
        if (s != VANN_OK) {
            cudaFree(rows);
            check(s);
        }
        return rows;
    }

    void patchGraph() {
        check(vann_patch_graph(h_, nullptr, nullptr));
        check(vann_consolidate(h_, nullptr));
    }

    void saveGraph(const std::string& path) { check(vann_save_graph(h_, path.c_str())); }

    vann_index* handle() const { return h_; }

   private:
    void create(uint64_t n) {
        vann_params vp{};
        vp.dim         = p_.dim;
        vp.degree      = p_.R;
        vp.build_L     = p_.L;
        vp.alpha       = p_.alpha;
        vp.capacity    = (uint64_t)(n * p_.capacity_factor) + 1;
        vp.max_visited = p_.max_visited;
        vp.max_reverse = p_.max_reverse;
        vp.flags       = p_.reference_quirks ? VANN_QUIRK_SKIP_BATCH_INDEX : 0u;
        vp.stores      = 0;
        check(vann_create(&vp, &h_));
    }

    VamanaParams p_;
    vann_index*  h_ = nullptr;
};

}  // namespace vann

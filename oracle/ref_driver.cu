// ref_driver.cu -- runs the reference's own CUDA GreedySearch and runVamana.
//
// TEST INFRASTRUCTURE ONLY: a second oracle.  Built by `make -C oracle ref` from
// the reference's sources where they lie (vamana/include/*.cuh, vamana/src/
// globals.cu, *_list_kernels.cu; nothing is copied) into oracle/_ref/.  Its
// compile-time constants are the reference's: D=128, R=64, L=199, medoid 5000,
// 10,000 records (vamana/include/constants.cuh:7-13).
//
//   ref_vamana search <graph.bin> <queries.f32> <n> <out_ids.u32>
//       greedySearch (search.cuh:226-367) over n queries; writes n x L worklist ids
//   ref_vamana time <graph.bin> <queries.f32> <n> <reps>
//       the same call reps times (after one untimed call); prints one line
//       "REFTIME <ms> <ms> ..." of wall time per call, each call bracketed by a
//       device synchronize (greedySearch allocates, launches four kernels per hop
//       and polls the host for termination, so its wall time is its cost)
//
// Only the search is driven.  The reference's build (runVamana) reads its
// reverse-index allocation without clearing it (vamana_impl.cuh:316-318): on
// memory that is not zero it would index past the 500-entry records, so it is
// not run on a shared GPU.  The build is pinned by the reference's golden graph
// instead (tests/test_oracle_golden.py).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "vamana.cuh"

using namespace FreshVamana;

static int do_search(const char* graph, const char* qpath, size_t n, const char* out) {
    auto g = initGraph<float>(graph);
    if (!g) return 2;
    std::vector<float> q(n * Consts::D_g);
    FILE*              f = fopen(qpath, "rb");
    if (!f || fread(q.data(), sizeof(float), q.size(), f) != q.size()) return 3;
    fclose(f);
    float* d_q = nullptr;
    gpuErrchk(cudaMalloc(&d_q, q.size() * sizeof(float)));
    gpuErrchk(cudaMemcpy(d_q, q.data(), q.size() * sizeof(float), cudaMemcpyHostToDevice));
    uint*  d_vis = nullptr;
    uint*  d_vcnt = nullptr;
    gpuErrchk(cudaMalloc(&d_vis, n * Consts::max_num_parents_per_query * sizeof(uint)));
    gpuErrchk(cudaMalloc(&d_vcnt, n * sizeof(uint)));
    gpuErrchk(cudaMemset(d_vcnt, 0, n * sizeof(uint)));
    uint* d_wl = greedySearch<float>(g->d_graph, nullptr, 0, d_q, d_vis, d_vcnt, (uint)n);
    std::vector<uint> wl(n * Consts::L_g);
    gpuErrchk(cudaMemcpy(wl.data(), d_wl, wl.size() * sizeof(uint), cudaMemcpyDeviceToHost));
    f = fopen(out, "wb");
    if (!f) return 4;
    fwrite(wl.data(), sizeof(uint), wl.size(), f);
    fclose(f);
    return 0;
}

static int do_time(const char* graph, const char* qpath, size_t n, int reps) {
    auto g = initGraph<float>(graph);
    if (!g) return 2;
    std::vector<float> q(n * Consts::D_g);
    FILE*              f = fopen(qpath, "rb");
    if (!f || fread(q.data(), sizeof(float), q.size(), f) != q.size()) return 3;
    fclose(f);
    float* d_q = nullptr;
    gpuErrchk(cudaMalloc(&d_q, q.size() * sizeof(float)));
    gpuErrchk(cudaMemcpy(d_q, q.data(), q.size() * sizeof(float), cudaMemcpyHostToDevice));
    uint* d_vis  = nullptr;
    uint* d_vcnt = nullptr;
    gpuErrchk(cudaMalloc(&d_vis, n * Consts::max_num_parents_per_query * sizeof(uint)));
    gpuErrchk(cudaMalloc(&d_vcnt, n * sizeof(uint)));
    std::vector<double> ms;
    for (int r = 0; r <= reps; ++r) {
        gpuErrchk(cudaMemset(d_vcnt, 0, n * sizeof(uint)));
        gpuErrchk(cudaDeviceSynchronize());
        const auto t0   = std::chrono::steady_clock::now();
        uint*      d_wl = greedySearch<float>(g->d_graph, nullptr, 0, d_q, d_vis, d_vcnt, (uint)n);
        gpuErrchk(cudaDeviceSynchronize());
        const auto t1 = std::chrono::steady_clock::now();
        gpuErrchk(cudaFree(d_wl));  // the caller owns the returned worklist
        if (r > 0) ms.push_back(std::chrono::duration<double, std::milli>(t1 - t0).count());
    }
    printf("REFTIME");
    for (double t : ms) printf(" %.4f", t);
    printf("\n");
    return 0;
}

int main(int argc, char** argv) {
    if (argc == 6 && std::string(argv[1]) == "search")
        return do_search(argv[2], argv[3], strtoull(argv[4], nullptr, 10), argv[5]);
    if (argc == 6 && std::string(argv[1]) == "time")
        return do_time(argv[2], argv[3], strtoull(argv[4], nullptr, 10), atoi(argv[5]));
    fprintf(stderr, "usage: %s search <graph.bin> <q.f32> <n> <out.u32>\n"
                    "       %s time <graph.bin> <q.f32> <n> <reps>\n", argv[0], argv[0]);
    return 1;
}

// rerank.cu -- the two passes around a search over a uint8 copy on a fitted grid
// (scalar quantization of float rows, graph_ops.cu launch_u8_grid).
//
// Before: the queries are mapped onto the grid and rounded, so the search kernels
// run their exact integer (dp4a) path on code distances, unchanged.
// After: the L candidates of each query are reranked with exact FP32 distances --
// the same distance code, key (distance, list position) and sort as the search
// kernels' in-kernel rerank -- or, without a rerank, the code distances are scaled
// back to the rows' units.
#include "common.cuh"
#include "kernels.h"

namespace vann {
namespace {

constexpr uint32_t kRerankWarps = 4;

__global__ void grid_queries_kernel(const float* q, uint64_t n, uint32_t D, const float* lo, float inv,
                                    float* out) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t d = (uint32_t)(i % D);
    out[i]           = fminf(fmaxf(rintf((q[i] - lo[d]) * inv), 0.f), 255.f);
}

// One warp per query: the list's ids, exact FP32 distances in gather rounds, a sort of
// (distance, position) keys in shared memory, the first k (or kq[q]) written out.
template <int DC>
__global__ void __launch_bounds__(kRerankWarps * 32) rerank_kernel(const float* vecs, const float* queries,
                                                                   uint64_t nq, uint32_t D, const uint32_t* cand,
                                                                   uint32_t L, uint32_t Lp, const uint32_t* kq,
                                                                   uint32_t k, uint32_t* out_ids, float* out_d) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int  GF   = Layout<StoreF32, DC>::kG;
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    uint64_t*      keys = reinterpret_cast<uint64_t*>(smem) + (size_t)wib * Lp;
    uint32_t*      ids  = reinterpret_cast<uint32_t*>(smem + 8ull * Lp * kRerankWarps) + (size_t)wib * Lp;
    for (uint64_t q = blockIdx.x * (uint64_t)kRerankWarps + wib; q < nq; q += (uint64_t)gridDim.x * kRerankWarps) {
        uint32_t n = 0;  // the list's entries (a prefix; kNone after it)
        for (uint32_t c0 = 0; c0 < L; c0 += 32u) {
            const uint32_t i  = c0 + lane;
            const uint32_t id = i < L ? __ldg(cand + q * L + i) : kNone;
            if (i < L) ids[i] = id;
            n += __popc(__ballot_sync(0xffffffffu, id != kNone));
        }
        __syncwarp();
        Query<StoreF32, DC> qf;
        load_query<StoreF32, DC>(qf, queries + q * D, D, lane);
        for (uint32_t g0 = 0; g0 < n; g0 += GF) {
            const int      gc = (int)min((uint32_t)GF, n - g0);
            const float    y  = dist_group<StoreF32, DC>(qf, vecs, nullptr, [&](int j) { return ids[g0 + j]; }, gc,
                                                         D, lane);
            const uint32_t vi = round_row_of_lane<StoreF32, DC>(lane);
            if (round_writer<StoreF32, DC>(lane) && (int)vi < gc) keys[g0 + vi] = make_key(y, g0 + vi);
        }
        __syncwarp();
        uint32_t ns = 32;
        while (ns < n) ns <<= 1;
        for (uint32_t i = n + lane; i < ns; i += 32u) keys[i] = ~0ull;
        __syncwarp();
        warp_bitonic_sort_smem(keys, ns, lane);
        const uint32_t kk = kq != nullptr ? min(__ldg(kq + q), k) : k;
        for (uint32_t t = lane; t < k; t += 32u) {
            const uint64_t o = q * k + t;
            if (t < n && t < kk) {
                out_ids[o] = ids[(uint32_t)keys[t]];
                out_d[o]   = key_dist(keys[t]);
            } else {
                out_ids[o] = kNone;
                out_d[o]   = __int_as_float(0x7f800000);
            }
        }
        __syncwarp();
    }
}

__global__ void scale_kernel(float* x, uint64_t n, float f) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) x[i] *= f;
}

template <int DC>
cudaError_t launch_rerank_dc(const float* vecs, const float* q, uint64_t nq, uint32_t D, const uint32_t* cand,
                             uint32_t L, const uint32_t* kq, uint32_t k, uint32_t* out_ids, float* out_d,
                             int num_sms, cudaStream_t st) {
    uint32_t Lp = 32;
    while (Lp < L) Lp <<= 1;
    const size_t smem = (size_t)kRerankWarps * Lp * (sizeof(uint64_t) + sizeof(uint32_t));
    auto         kern = rerank_kernel<DC>;
    cudaError_t  e    = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    uint64_t grid = (nq + kRerankWarps - 1) / kRerankWarps;
    const uint64_t cap = (uint64_t)num_sms * 8u;
    if (grid > cap) grid = cap;
    kern<<<(unsigned)grid, kRerankWarps * 32, smem, st>>>(vecs, q, nq, D, cand, L, Lp, kq, k, out_ids, out_d);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_grid_queries(const float* q, uint64_t nq, uint32_t D, const float* lo, float inv, float* out,
                                cudaStream_t st) {
    const uint64_t n = nq * D;
    if (n == 0) return cudaSuccess;
    grid_queries_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(q, n, D, lo, inv, out);
    return cudaGetLastError();
}

cudaError_t launch_rerank(const float* vecs, const float* q, uint64_t nq, uint32_t D, const uint32_t* cand,
                          uint32_t L, const uint32_t* kq, uint32_t k, uint32_t* out_ids, float* out_d,
                          int num_sms, cudaStream_t st) {
    if (nq == 0) return cudaSuccess;
    if (L == 0 || L > 1024 || D % 4 != 0) return cudaErrorInvalidValue;
    if (D <= 128) return launch_rerank_dc<0>(vecs, q, nq, D, cand, L, kq, k, out_ids, out_d, num_sms, st);
    if (D <= 256) return launch_rerank_dc<1>(vecs, q, nq, D, cand, L, kq, k, out_ids, out_d, num_sms, st);
    if (D <= 512) return launch_rerank_dc<2>(vecs, q, nq, D, cand, L, kq, k, out_ids, out_d, num_sms, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_scale(float* x, uint64_t n, float f, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, n, f);
    return cudaGetLastError();
}

}  // namespace vann

// pq.cu -- product-quantized traversal codes (VANN_STORE_PQ).
//
// Product quantization (Jegou, Douze, Schmid, "Product quantization for nearest
// neighbor search", IEEE TPAMI 33(1), 2011): a row is cut into D / 8 subspaces of
// 8 dimensions, and each piece is replaced by the index of its nearest of 256
// centroids, learnt per subspace by k-means (Lloyd's algorithm) on a sample of the
// rows.  A search compares a query with a row through a table of the query's
// squared distances to every centroid (build_pq_lut, common.cuh): one table lookup
// per code byte.  That is the compressed traversal of BANG, whose distance kernel
// reads such per-query tables (bang_exact/src/parANN.cu:1107-1157; the reference's
// copy of BANG keeps its table allocations commented out, :264-265, :350-351).  The
// exact FP32 rerank of the final worklist gives exact returned distances.
//
// Training is deterministic: the initial centroids are evenly spaced sample rows,
// an assignment keeps the lowest centroid index on ties, and each centroid's sum is
// taken in sample order, so the same rows always give the same codebook.
#include "common.cuh"
#include "kernels.h"

namespace vann {
namespace {

constexpr uint32_t kSampleMax = 65536;  // training rows
constexpr int      kIters     = 12;     // Lloyd iterations

__global__ void pq_gather_kernel(const float* vecs, uint64_t n, uint32_t D, uint32_t ns, float* sample) {
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint32_t q = D / 4;
    if (t >= (uint64_t)ns * q) return;
    const uint64_t s = t / q, c = t % q;
    const uint64_t r = s * n / ns;  // evenly spaced rows
    reinterpret_cast<float4*>(sample + s * D)[c] = __ldg(reinterpret_cast<const float4*>(vecs + r * D) + c);
}

// centroid k of every subspace starts as sample row k * ns / 256 (k mod ns when ns < 256)
__global__ void pq_init_kernel(const float* sample, uint32_t ns, uint32_t D, float* cb) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;  // over M * 256 * 8
    const uint32_t M = D / kPqSub;
    if (t >= M * kPqK * kPqSub) return;
    const uint32_t m = t / (kPqK * kPqSub), k = (t / kPqSub) % kPqK, d = t % kPqSub;
    const uint64_t s = ns >= kPqK ? (uint64_t)k * ns / kPqK : k % ns;
    cb[t]            = sample[s * D + m * kPqSub + d];
}

// nearest centroid of subspace blockIdx.y for rows (sample rows, or the index's rows
// first + i, or ids[i]); lowest index on ties.  The subspace's 256 x 8 centroids
// are staged in shared memory and read as broadcasts.
__global__ void __launch_bounds__(256) pq_assign_kernel(const float* rows_base, uint64_t first, const uint32_t* ids,
                                                        uint64_t nrows, uint32_t D, const float* cb, uint8_t* out,
                                                        uint64_t out_first) {
    __shared__ float4 c[kPqK * 2];
    const uint32_t m = blockIdx.y;
    const uint32_t M = D / kPqSub;
    for (uint32_t i = threadIdx.x; i < kPqK * 2; i += blockDim.x)
        c[i] = __ldg(reinterpret_cast<const float4*>(cb + (uint64_t)m * kPqK * kPqSub) + i);
    __syncthreads();
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const uint64_t r  = ids != nullptr ? ids[i] : first + i;
    const float4   xa = __ldg(reinterpret_cast<const float4*>(rows_base + r * D + m * kPqSub));
    const float4   xb = __ldg(reinterpret_cast<const float4*>(rows_base + r * D + m * kPqSub) + 1);
    float          best = __int_as_float(0x7f800000);
    uint32_t       bk   = 0;
    for (uint32_t k = 0; k < kPqK; ++k) {
        const float4 a = c[2 * k], b = c[2 * k + 1];
        float        d = 0.f;
        d              = sqdiff(xa.x, a.x, d);
        d              = sqdiff(xa.y, a.y, d);
        d              = sqdiff(xa.z, a.z, d);
        d              = sqdiff(xa.w, a.w, d);
        d              = sqdiff(xb.x, b.x, d);
        d              = sqdiff(xb.y, b.y, d);
        d              = sqdiff(xb.z, b.z, d);
        d              = sqdiff(xb.w, b.w, d);
        if (d < best) {
            best = d;
            bk   = k;
        }
    }
    const uint64_t o = ids != nullptr ? (uint64_t)ids[i] : out_first + i;
    out[o * M + m]   = (uint8_t)bk;
}

// New centroids: block (m, kb) holds centroids kb * 256 / KPB .. of subspace m, one
// thread per (centroid, dimension); every thread walks the sample in order and adds
// the rows assigned to its centroid in FP64, so the sums are the same on every run.
// A centroid without rows keeps its position.
constexpr uint32_t kUpdThreads = 256;                    // threads per block
constexpr uint32_t kUpdCent    = kUpdThreads / kPqSub;   // centroids per block (32)
__global__ void __launch_bounds__(kUpdThreads) pq_update_kernel(const float* sample, uint32_t ns, uint32_t D,
                                                                const uint8_t* assign, float* cb) {
    const uint32_t m = blockIdx.y;
    const uint32_t M = D / kPqSub;
    const uint32_t k = blockIdx.x * kUpdCent + threadIdx.x / kPqSub;
    const uint32_t d = threadIdx.x % kPqSub;
    double         sum = 0.0;
    uint32_t       cnt = 0;
    for (uint32_t s = 0; s < ns; ++s) {
        if (assign[(uint64_t)s * M + m] == k) {
            sum += (double)sample[(uint64_t)s * D + m * kPqSub + d];
            ++cnt;
        }
    }
    if (cnt > 0) cb[((uint64_t)m * kPqK + k) * kPqSub + d] = (float)(sum / (double)cnt);
}

// largest centroid norm per subspace (the table scale's bound), one warp per subspace
__global__ void pq_cnorm_kernel(uint32_t D, const float* cb, float* cnorm) {
    const uint32_t m    = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const uint32_t lane = threadIdx.x & 31u;
    if (m >= D / kPqSub) return;
    float best = 0.f;
    for (uint32_t k = lane; k < kPqK; k += 32) {
        const float* c = cb + ((uint64_t)m * kPqK + k) * kPqSub;
        float        s = 0.f;
        for (uint32_t d = 0; d < kPqSub; ++d) s = fmaf(c[d], c[d], s);
        best = fmaxf(best, sqrtf(s));
    }
    for (int o = 16; o >= 1; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if (lane == 0) cnorm[m] = best;
}

size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

}  // namespace

size_t pq_train_ws_bytes(uint64_t n, uint32_t D) {
    const uint64_t ns = n < kSampleMax ? n : kSampleMax;
    const uint32_t M  = D / kPqSub;
    return al256(sizeof(float) * ns * D) + al256(ns * M);
}

cudaError_t launch_pq_train(const float* vecs, uint64_t n, uint32_t D, float* cb, float* cnorm, void* ws,
                            cudaStream_t st) {
    if (n == 0 || D % 128 != 0) return cudaErrorInvalidValue;
    const uint32_t ns = (uint32_t)(n < kSampleMax ? n : kSampleMax);
    const uint32_t M  = D / kPqSub;
    float*         sample = static_cast<float*>(ws);
    uint8_t*       assign = static_cast<uint8_t*>(ws) + al256(sizeof(float) * (uint64_t)ns * D);

    cudaError_t    e   = cudaSuccess;
    const uint64_t g4  = (uint64_t)ns * (D / 4);
    pq_gather_kernel<<<(unsigned)((g4 + 255) / 256), 256, 0, st>>>(vecs, n, D, ns, sample);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const uint32_t ncb = M * kPqK * kPqSub;
    pq_init_kernel<<<(ncb + 255) / 256, 256, 0, st>>>(sample, ns, D, cb);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const dim3 ga((ns + 255) / 256, M);
    const dim3 gu(kPqK / kUpdCent, M);
    for (int it = 0; it < kIters; ++it) {
        pq_assign_kernel<<<ga, 256, 0, st>>>(sample, 0, nullptr, ns, D, cb, assign, 0);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        pq_update_kernel<<<gu, kUpdThreads, 0, st>>>(sample, ns, D, assign, cb);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    pq_cnorm_kernel<<<(M + 3) / 4, 128, 0, st>>>(D, cb, cnorm);
    return cudaGetLastError();
}

cudaError_t launch_pq_encode(const float* vecs, uint64_t first, uint64_t rows, const uint32_t* ids, uint32_t D,
                             const float* cb, uint8_t* codes, cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    const dim3 g((unsigned)((rows + 255) / 256), D / kPqSub);
    pq_assign_kernel<<<g, 256, 0, st>>>(vecs, first, ids, rows, D, cb, codes, first);
    return cudaGetLastError();
}

}  // namespace vann

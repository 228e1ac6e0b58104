// graph_ops.cu -- small HBM-bound kernels around the search and prune kernels:
// random start graph, storage conversion, tombstones, medoid, reverse-edge
// lists, delete-by-vector and delete-consolidation candidates.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <mutex>

#include "../../include/vann.h"
#include "common.cuh"
#include "kernels.h"

namespace vann {

// SplitMix64 finaliser (Steele, Lea, Flood 2014)
__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    uint64_t z = x + 0x9e3779b97f4a7c15ull;
    z          = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z          = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Random R-regular start graph over ids first .. first+n-1 (the reference reads
// one from a file, utils.cuh:113-148).  Slot j of node i points at
// first + (i + 1 + h % (n - 1)) % n with h = splitmix64(seed ^ (i * R + j)).
__global__ void random_graph_kernel(uint32_t* deg, uint32_t* adj, uint32_t* adj_h, uint64_t first,
                                    uint64_t n, uint32_t R, uint64_t seed) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= n * R) return;
    uint64_t i = t / R, j = t % R;
    uint32_t v = 0;
    if (n > 1) {
        uint64_t h = splitmix64(seed ^ (i * R + j));
        v          = (uint32_t)(first + (i + 1 + h % (n - 1)) % n);
    }
    adj[(first + i) * R + j]   = v;
    adj_h[(first + i) * R + j] = bloom_pack(v);
    if (j == 0) deg[first + i] = n > 1 ? R : 0u;
}

cudaError_t launch_random_graph(uint32_t* deg, uint32_t* adj, uint32_t* adj_h, uint64_t first,
                                uint64_t n, uint32_t R, uint64_t seed, cudaStream_t st) {
    uint64_t total = n * R;
    if (total == 0) return cudaSuccess;
    random_graph_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(deg, adj, adj_h, first, n, R,
                                                                        seed);
    return cudaGetLastError();
}

__global__ void hash_rows_kernel(const uint32_t* adj, uint32_t* adj_h, uint64_t total) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t < total) adj_h[t] = bloom_pack(adj[t]);
}
cudaError_t launch_hash_rows(const uint32_t* adj, uint32_t* adj_h, uint64_t n, uint32_t R,
                             cudaStream_t st) {
    uint64_t total = n * R;
    if (total == 0) return cudaSuccess;
    hash_rows_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(adj, adj_h, total);
    return cudaGetLastError();
}

// FP32 rows -> traversal copies.  FP8: scale = amax / 448 per row (e4m3 max
// finite 448), codes = satfinite(x / scale).  U8: round to nearest, clamp.
__global__ void convert_kernel(const float* src, void* dst, float* scale, uint64_t rows, uint32_t D,
                               int store, uint32_t* inexact) {
    uint64_t r    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (r >= rows) return;
    const float* s = src + r * D;
    if (store == 1) {
        __nv_bfloat16* d = static_cast<__nv_bfloat16*>(dst) + r * D;
        for (uint32_t i = lane; i < D; i += 32) d[i] = __float2bfloat16_rn(s[i]);
    } else if (store == 2) {
        float amax = 0.f;
        for (uint32_t i = lane; i < D; i += 32) amax = fmaxf(amax, fabsf(s[i]));
        for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        float sc  = amax > 0.f ? amax / 448.f : 1.f;
        float inv = 1.f / sc;
        uint8_t* d = static_cast<uint8_t*>(dst) + r * D;
        for (uint32_t i = lane; i < D; i += 32)
            d[i] = (uint8_t)__nv_cvt_float_to_fp8(s[i] * inv, __NV_SATFINITE, __NV_E4M3);
        if (lane == 0) scale[r] = sc;
    } else if (store == 3) {
        uint8_t* d   = static_cast<uint8_t*>(dst) + r * D;
        bool     off = false;
        for (uint32_t i = lane; i < D; i += 32) {
            float v = rintf(s[i]);
            v       = fminf(fmaxf(v, 0.f), 255.f);
            d[i]    = (uint8_t)v;
            off |= !(v == s[i]);
        }
        if (__any_sync(0xffffffffu, off) && lane == 0) atomicOr(inexact, 1u);
    }
}

cudaError_t launch_convert(const float* src, void* dst, float* scale, uint64_t rows, uint32_t D,
                           int store, uint32_t* inexact, cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    convert_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(src, dst, scale, rows, D, store, inexact);
    return cudaGetLastError();
}

// Same conversion for rows scattered over an id list (inserts into reused ids):
// one warp per listed row, the row's traversal copy rewritten from its FP32 row.
__global__ void convert_ids_kernel(const float* vecs, const uint32_t* ids, uint64_t n, void* dst,
                                   float* scale, uint32_t D, int store, uint32_t* inexact) {
    uint64_t i    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (i >= n) return;
    const uint64_t r = ids[i];
    const float*   s = vecs + r * D;
    if (store == 1) {
        __nv_bfloat16* d = static_cast<__nv_bfloat16*>(dst) + r * D;
        for (uint32_t k = lane; k < D; k += 32) d[k] = __float2bfloat16_rn(s[k]);
    } else if (store == 2) {
        float amax = 0.f;
        for (uint32_t k = lane; k < D; k += 32) amax = fmaxf(amax, fabsf(s[k]));
        for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
        float    sc  = amax > 0.f ? amax / 448.f : 1.f;
        float    inv = 1.f / sc;
        uint8_t* d   = static_cast<uint8_t*>(dst) + r * D;
        for (uint32_t k = lane; k < D; k += 32)
            d[k] = (uint8_t)__nv_cvt_float_to_fp8(s[k] * inv, __NV_SATFINITE, __NV_E4M3);
        if (lane == 0) scale[r] = sc;
    } else if (store == 3) {
        uint8_t* d   = static_cast<uint8_t*>(dst) + r * D;
        bool     off = false;
        for (uint32_t k = lane; k < D; k += 32) {
            const float v = fminf(fmaxf(rintf(s[k]), 0.f), 255.f);
            d[k]          = (uint8_t)v;
            off |= !(v == s[k]);
        }
        if (__any_sync(0xffffffffu, off) && lane == 0) atomicOr(inexact, 1u);
    }
}
cudaError_t launch_convert_ids(const float* vecs, const uint32_t* ids, uint64_t n, void* dst, float* scale,
                               uint32_t D, int store, uint32_t* inexact, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    convert_ids_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(vecs, ids, n, dst, scale, D, store, inexact);
    return cudaGetLastError();
}

__global__ void iota_kernel(uint32_t* out, uint64_t n, uint32_t first) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < n) out[i] = first + (uint32_t)i;
}
cudaError_t launch_iota(uint32_t* out, uint64_t n, uint32_t first, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    iota_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, first);
    return cudaGetLastError();
}

__global__ void set_bits_kernel(uint32_t* bits, const uint32_t* ids, uint64_t n, uint64_t limit) {
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t id = ids[i];
    if (id < limit) atomicOr(bits + (id >> 5), 1u << (id & 31u));
}
cudaError_t launch_set_bits(uint32_t* bits, const uint32_t* ids, uint64_t n, uint64_t limit,
                            cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    set_bits_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(bits, ids, n, limit);
    return cudaGetLastError();
}

// Medoid = argmin_i ||x_i - mean||^2 in FP64, smallest id on ties
// (parth/tools/vamana.py:25-29).  mean_ws: D doubles; best_ws: [min bits, id].
__global__ void col_sum_kernel(const float* vecs, uint64_t n, uint32_t D, double* sum) {
    uint32_t d  = threadIdx.x + blockIdx.y * blockDim.x;
    if (d >= D) return;
    uint64_t r0 = blockIdx.x * (uint64_t)1024;
    uint64_t r1 = n < r0 + 1024 ? n : r0 + 1024;
    double   s  = 0.0;
    for (uint64_t r = r0; r < r1; ++r) s += (double)vecs[r * D + d];
    atomicAdd(sum + d, s);
}
__global__ void medoid_dist_kernel(const float* vecs, uint64_t n, uint32_t D, const double* sum,
                                   unsigned long long* best, int pass) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    double s = 0.0;
    for (uint32_t d = 0; d < D; ++d) {
        double t = (double)vecs[r * D + d] - sum[d] / (double)n;
        s += t * t;
    }
    unsigned long long bits = (unsigned long long)__double_as_longlong(s);
    if (pass == 0)
        atomicMin(best, bits);
    else if (bits == best[0])
        atomicMin(best + 1, (unsigned long long)r);
}
cudaError_t launch_medoid(const float* vecs, uint64_t n, uint32_t D, double* mean_ws,
                          unsigned long long* best_ws, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(mean_ws, 0, sizeof(double) * D, st);
    if (e != cudaSuccess) return e;
    unsigned long long init[2] = {~0ull, ~0ull};
    e = cudaMemcpyAsync(best_ws, init, sizeof(init), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    dim3 g((unsigned)((n + 1023) / 1024), (D + 127) / 128);
    col_sum_kernel<<<g, 128, 0, st>>>(vecs, n, D, mean_ws);
    medoid_dist_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(vecs, n, D, mean_ws, best_ws, 0);
    medoid_dist_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(vecs, n, D, mean_ws, best_ws, 1);
    return cudaGetLastError();
}

// Reverse edges of a pruned batch: keys = target, vals = source, padded slots
// get target UINT32_MAX.  counts[target] counts the valid ones.
__global__ void edges_kernel(const uint32_t* nodes, uint64_t n_nodes, const uint32_t* deg,
                             const uint32_t* adj, uint32_t R, uint32_t* keys, uint32_t* vals,
                             uint32_t* counts) {
    uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (t >= n_nodes * R) return;
    uint64_t b    = t / R;
    uint32_t j    = (uint32_t)(t % R);
    uint32_t node = nodes[b];
    if (j < deg[node]) {
        uint32_t tg = adj[(uint64_t)node * R + j];
        keys[t]     = tg;
        vals[t]     = node;
        if (counts != nullptr) atomicAdd(counts + tg, 1u);
    } else {
        keys[t] = kNone;
        vals[t] = kNone;
    }
}
cudaError_t launch_edges(const uint32_t* nodes, uint64_t n_nodes, const uint32_t* deg,
                         const uint32_t* adj, uint32_t R, uint32_t* keys, uint32_t* vals,
                         uint32_t* counts, cudaStream_t st) {
    uint64_t total = n_nodes * R;
    if (total == 0) return cudaSuccess;
    edges_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(nodes, n_nodes, deg, adj, R, keys,
                                                                 vals, counts);
    return cudaGetLastError();
}

// Delete by exact vector match (findPointsKernel, kernels.cuh:905-933): warp
// per (query, 32-row tile); out[q] = smallest matching live id or -1.
__global__ void find_vectors_kernel(const float* vecs, uint64_t n, uint32_t D, const float* q,
                                    uint64_t nq, const uint32_t* tomb, int32_t* out) {
    uint64_t qi   = blockIdx.y;
    uint64_t r    = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (qi >= nq || r >= n) return;
    if (tomb && ((tomb[r >> 5] >> (r & 31u)) & 1u)) return;
    const float4* a = reinterpret_cast<const float4*>(vecs + r * D);
    const float4* b = reinterpret_cast<const float4*>(q + qi * D);
    for (uint32_t c = 0; c < D / 4; ++c) {
        float4 x = __ldg(a + c), y = __ldg(b + c);
        if (x.x != y.x || x.y != y.y || x.z != y.z || x.w != y.w) return;
    }
    atomicMin(reinterpret_cast<unsigned int*>(out + qi), (unsigned int)r);
}
cudaError_t launch_find_vectors(const float* vecs, uint64_t n, uint32_t D, const float* q,
                                uint64_t nq, const uint32_t* tomb, int32_t* out, cudaStream_t st) {
    if (nq == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(out, 0xff, sizeof(int32_t) * nq, st);
    if (e != cudaSuccess || n == 0) return e;
    dim3 g((unsigned)((n + 255) / 256), (unsigned)nq);
    find_vectors_kernel<<<g, 256, 0, st>>>(vecs, n, D, q, nq, tomb, out);
    return cudaGetLastError();
}

// Delete consolidation candidates (FreshDiskANN, Singh et al. 2021, Alg. 4):
// for every live node p with a deleted out-neighbour, C = (out(p) \ D) U
// (out(d) \ D for deleted d in out(p)), minus p, first occurrence kept, capped.
// One warp per node; p is appended to node_list.  cand_d receives dist(p, c).
__global__ void consolidate_candidates_kernel(const uint32_t* deg, const uint32_t* adj, uint32_t R,
                                              const uint32_t* tomb, uint64_t n,
                                              uint32_t* node_list, uint32_t* n_list,
                                              uint32_t* cand, uint32_t* cand_n, float* cand_d,
                                              const float* vecs, uint32_t D, uint32_t cap) {
    uint64_t p    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (p >= n) return;
    auto dead = [&](uint32_t id) { return (tomb[id >> 5] >> (id & 31u)) & 1u; };
    if (dead((uint32_t)p)) return;
    uint32_t dg  = min(deg[p], R);
    bool     any = false;
    for (uint32_t j = lane; j < dg; j += 32) any |= dead(adj[p * R + j]) != 0;
    if (!__any_sync(0xffffffffu, any)) return;
    uint32_t slot = 0;
    if (lane == 0) slot = atomicAdd(n_list, 1u);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    if (lane == 0) node_list[slot] = (uint32_t)p;
    uint32_t* c   = cand + (uint64_t)slot * cap;
    uint32_t  cnt = 0;
    // serial over out(p) in order keeps the candidate order deterministic
    for (uint32_t j = 0; j < dg; ++j) {
        uint32_t v = adj[p * R + j];
        if (!dead(v)) {
            bool dup = false;
            for (uint32_t t = lane; t < cnt; t += 32) dup |= c[t] == v;
            dup = __any_sync(0xffffffffu, dup);
            if (!dup && v != (uint32_t)p && cnt < cap) {
                if (lane == 0) c[cnt] = v;
                ++cnt;
            }
            __syncwarp();
        } else {
            uint32_t dd = min(deg[v], R);
            for (uint32_t k = 0; k < dd; ++k) {
                uint32_t u = adj[(uint64_t)v * R + k];
                if (dead(u) || u == (uint32_t)p) continue;
                bool dup = false;
                for (uint32_t t = lane; t < cnt; t += 32) dup |= c[t] == u;
                dup = __any_sync(0xffffffffu, dup);
                if (!dup && cnt < cap) {
                    if (lane == 0) c[cnt] = u;
                    ++cnt;
                }
                __syncwarp();
            }
        }
    }
    // distances to p
    for (uint32_t t = 0; t < cnt; ++t) {
        const float* a = vecs + (uint64_t)p * D;
        const float* b = vecs + (uint64_t)c[t] * D;
        float        s = 0.f;
        for (uint32_t d = lane; d < D; d += 32) {
            float x = a[d] - b[d];
            s       = fmaf(x, x, s);
        }
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) cand_d[(uint64_t)slot * cap + t] = s;
    }
    if (lane == 0) cand_n[slot] = cnt;
}
cudaError_t launch_consolidate_candidates(const uint32_t* deg, const uint32_t* adj, uint32_t R,
                                          const uint32_t* tomb, uint64_t n, uint32_t* node_list,
                                          uint32_t* n_list, uint32_t* cand, uint32_t* cand_n,
                                          float* cand_d, const float* vecs, uint32_t D,
                                          uint32_t cap, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    consolidate_candidates_kernel<<<(unsigned)((n + 3) / 4), 128, 0, st>>>(
        deg, adj, R, tomb, n, node_list, n_list, cand, cand_n, cand_d, vecs, D, cap);
    return cudaGetLastError();
}

}  // namespace vann

// ---------------------------------------------------------------- allocation-free medoid
// Entry-point selection (the medoid above) for callers that must not allocate
// device memory.  Its scratch -- the D column sums (FP64) and the argmin word
// pair -- lives in this file-scope device array instead of memory the library
// would cudaMalloc: up to kNoAllocMaxDim dimensions, 32 KiB + 256 B, held by
// every device that loads the library until the process exits.
namespace {
constexpr uint32_t kNoAllocMaxDim = 4096;
constexpr size_t   kNoAllocSumBytes = sizeof(double) * kNoAllocMaxDim;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocSumBytes + 256];

__global__ void medoid_result_kernel(const unsigned long long* best, uint32_t* out) {
    *out = (uint32_t)best[1];
}

// device address of g_noalloc_scratch per device, resolved once per device
std::mutex g_noalloc_mu;
void*      g_noalloc_addr[256] = {};
}  // namespace

extern "C" vann_status vann_medoid_noalloc(const float* d_vecs, uint64_t n, uint32_t dim,
                                           uint32_t* d_medoid_out, void* stream) {
    if (d_vecs == nullptr || d_medoid_out == nullptr || n == 0 || dim == 0) {
        vann::set_last_error("vann_medoid_noalloc: null pointer or empty input");
        return VANN_ERR_INVALID;
    }
    if (dim > kNoAllocMaxDim) {
        vann::set_last_error("vann_medoid_noalloc: dim exceeds the fixed scratch maximum of 4096");
        return VANN_ERR_UNSUPPORTED;
    }
    if (n >= 0xffffffffull) {
        vann::set_last_error("vann_medoid_noalloc: n must be below 2^32");
        return VANN_ERR_UNSUPPORTED;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        vann::set_last_error("vann_medoid_noalloc: no current CUDA device");
        return VANN_ERR_CUDA;
    }
    void* base = nullptr;
    {
        // set-up on the first call on this device (with the device current):
        // the host-side symbol is only a stand-in, the kernels need the device
        // address, which cudaGetSymbolAddress resolves here
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (g_noalloc_addr[dev] == nullptr) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) {
                vann::set_last_error("vann_medoid_noalloc: cudaGetSymbolAddress failed");
                return VANN_ERR_CUDA;
            }
            g_noalloc_addr[dev] = p;
        }
        base = g_noalloc_addr[dev];
    }
    cudaStream_t        st   = static_cast<cudaStream_t>(stream);
    double*             sums = static_cast<double*>(base);
    unsigned long long* best = reinterpret_cast<unsigned long long*>(static_cast<char*>(base) + kNoAllocSumBytes);
    // the array keeps the previous call's contents: clear what must start fresh
    if (cudaMemsetAsync(sums, 0, sizeof(double) * dim, st) != cudaSuccess ||
        cudaMemsetAsync(best, 0xff, 2 * sizeof(unsigned long long), st) != cudaSuccess) {
        vann::set_last_error("vann_medoid_noalloc: clearing the scratch failed");
        return VANN_ERR_CUDA;
    }
    dim3 g((unsigned)((n + 1023) / 1024), (dim + 127) / 128);
    vann::col_sum_kernel<<<g, 128, 0, st>>>(d_vecs, n, dim, sums);
    vann::medoid_dist_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_vecs, n, dim, sums, best, 0);
    vann::medoid_dist_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_vecs, n, dim, sums, best, 1);
    medoid_result_kernel<<<1, 1, 0, st>>>(best, d_medoid_out);
    if (cudaGetLastError() != cudaSuccess) {
        vann::set_last_error("vann_medoid_noalloc: kernel launch failed");
        return VANN_ERR_CUDA;
    }
    return VANN_OK;
}


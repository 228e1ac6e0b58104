// graph_ops.cu -- small HBM-bound kernels around the search and prune kernels:
// random start graph, storage conversion, tombstones, medoid, reverse-edge
// lists, delete-by-vector and delete-consolidation candidates.
#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include <mutex>
#include <string>

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
// One row's e4m3 codes (one warp): the row is centred (row - center), s = amax / 448
// of the centred row, codes = centred row / s rounded to e4m3 (saturating), and
// beside s the squared norm of the decoded codes times s^2, which the traversal
// distance adds once per row.  Centring uses the format's sign bit for rows that
// are all non-negative, halving the scale and so the rounding error.
__device__ void fp8_row(const float* src, uint8_t* d, float2* scale, const float* center, uint32_t D,
                        uint32_t lane) {
    float amax = 0.f;
    for (uint32_t i = lane; i < D; i += 32) amax = fmaxf(amax, fabsf(src[i] - center[i]));
    for (int o = 16; o; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const float sc  = amax > 0.f ? amax / 448.f : 1.f;
    const float inv = 1.f / sc;
    float       cc  = 0.f;
    for (uint32_t i = lane; i < D; i += 32) {
        const __nv_fp8_storage_t c = __nv_cvt_float_to_fp8((src[i] - center[i]) * inv, __NV_SATFINITE, __NV_E4M3);
        d[i]                       = (uint8_t)c;
        const __half_raw h         = __nv_cvt_fp8_to_halfraw(c, __NV_E4M3);
        const float      v         = __half2float(*reinterpret_cast<const __half*>(&h));
        cc                         = fmaf(v, v, cc);
    }
    for (int o = 16; o; o >>= 1) cc += __shfl_xor_sync(0xffffffffu, cc, o);
    if (lane == 0) *scale = make_float2(sc, sc * sc * cc);
}

// uint8 code of value x: on the identity grid (lo == nullptr) the value itself,
// rounded and clamped; on a fitted grid round((x - lo[i]) * inv), clamped.
__device__ __forceinline__ float u8_code(float x, const float* lo, float inv, uint32_t i) {
    const float v = lo != nullptr ? rintf((x - lo[i]) * inv) : rintf(x);
    return fminf(fmaxf(v, 0.f), 255.f);
}

__global__ void convert_kernel(const float* src, void* dst, float2* scale, const float* center, float inv,
                               uint64_t rows, uint32_t D, int store, uint32_t* inexact) {
    uint64_t r    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (r >= rows) return;
    const float* s = src + r * D;
    if (store == 1) {
        __nv_bfloat16* d = static_cast<__nv_bfloat16*>(dst) + r * D;
        for (uint32_t i = lane; i < D; i += 32) d[i] = __float2bfloat16_rn(s[i]);
    } else if (store == 2) {
        fp8_row(s, static_cast<uint8_t*>(dst) + r * D, scale + r, center, D, lane);
    } else if (store == 3) {
        uint8_t* d   = static_cast<uint8_t*>(dst) + r * D;
        bool     off = center != nullptr;  // a fitted grid is approximate
        for (uint32_t i = lane; i < D; i += 32) {
            const float v = u8_code(s[i], center, inv, i);
            d[i]          = (uint8_t)v;
            off |= !(v == s[i]);
        }
        if (__any_sync(0xffffffffu, off) && lane == 0) atomicOr(inexact, 1u);
    }
}

cudaError_t launch_convert(const float* src, void* dst, float2* scale, const float* center, float inv,
                           uint64_t rows, uint32_t D, int store, uint32_t* inexact, cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    convert_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(src, dst, scale, center, inv, rows, D, store,
                                                               inexact);
    return cudaGetLastError();
}

// Same conversion for rows scattered over an id list (inserts into reused ids):
// one warp per listed row, the row's traversal copy rewritten from its FP32 row.
__global__ void convert_ids_kernel(const float* vecs, const uint32_t* ids, uint64_t n, void* dst,
                                   float2* scale, const float* center, float inv, uint32_t D, int store,
                                   uint32_t* inexact) {
    uint64_t i    = blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5);
    uint32_t lane = threadIdx.x & 31u;
    if (i >= n) return;
    const uint64_t r = ids[i];
    const float*   s = vecs + r * D;
    if (store == 1) {
        __nv_bfloat16* d = static_cast<__nv_bfloat16*>(dst) + r * D;
        for (uint32_t k = lane; k < D; k += 32) d[k] = __float2bfloat16_rn(s[k]);
    } else if (store == 2) {
        fp8_row(s, static_cast<uint8_t*>(dst) + r * D, scale + r, center, D, lane);
    } else if (store == 3) {
        uint8_t* d   = static_cast<uint8_t*>(dst) + r * D;
        bool     off = center != nullptr;
        for (uint32_t k = lane; k < D; k += 32) {
            const float v = u8_code(s[k], center, inv, k);
            d[k]          = (uint8_t)v;
            off |= !(v == s[k]);
        }
        if (__any_sync(0xffffffffu, off) && lane == 0) atomicOr(inexact, 1u);
    }
}
cudaError_t launch_convert_ids(const float* vecs, const uint32_t* ids, uint64_t n, void* dst, float2* scale,
                               const float* center, float inv, uint32_t D, int store, uint32_t* inexact,
                               cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    convert_ids_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(vecs, ids, n, dst, scale, center, inv, D, store,
                                                                inexact);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- uint8 grid
// The uint8 copy's grid, fitted to rows 0 .. n-1.  When every value is an integer
// in [0, 255] the grid is the identity and the copy is exact.  Otherwise every
// dimension gets its own offset lo[i] (the column minimum) and all share one
// scale s = max_i (max_i - lo[i]) / 255, so a squared distance on the codes is the
// squared distance on the rows divided by s^2 (up to rounding): traversal orders
// them alike, and s^2 brings the code distance back to the rows' units.
// ws (u8_grid_ws_bytes): per column the ordered bits of the minimum and maximum,
// then the off-grid flag.  grid out: {affine (0 / 1 as float), s, 1 / s}.

// order-preserving map of a float onto uint32 (ascending floats -> ascending words)
__device__ __forceinline__ uint32_t ord_bits(float x) {
    const uint32_t b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_float(uint32_t w) {
    return __uint_as_float((w & 0x80000000u) ? (w & 0x7fffffffu) : ~w);
}

__global__ void u8_minmax_kernel(const float* vecs, uint64_t n, uint32_t D, uint32_t* mn, uint32_t* mx,
                                 uint32_t* off) {
    const uint32_t d = threadIdx.x + blockIdx.y * blockDim.x;
    if (d >= D) return;
    const uint64_t r0 = blockIdx.x * (uint64_t)1024;
    const uint64_t r1 = n < r0 + 1024 ? n : r0 + 1024;
    uint32_t       lo = 0xffffffffu, hi = 0u;
    bool           bad = false;
    for (uint64_t r = r0; r < r1; ++r) {
        const float x = vecs[r * D + d];
        lo            = min(lo, ord_bits(x));
        hi            = max(hi, ord_bits(x));
        bad |= !(x >= 0.f && x <= 255.f && rintf(x) == x);
    }
    atomicMin(mn + d, lo);
    atomicMax(mx + d, hi);
    if (bad) atomicOr(off, 1u);
}

// one block: lo[] and grid[] from the column bounds
__global__ void u8_grid_kernel(const uint32_t* mn, const uint32_t* mx, const uint32_t* off, uint32_t D,
                               float* lo, float* grid) {
    __shared__ float red[32];
    const bool affine = *off != 0u;
    float      range  = 0.f;
    for (uint32_t d = threadIdx.x; d < D; d += blockDim.x) {
        const float a = ord_float(mn[d]);
        lo[d]         = affine ? a : 0.f;
        range         = fmaxf(range, ord_float(mx[d]) - a);
    }
    for (int o = 16; o; o >>= 1) range = fmaxf(range, __shfl_xor_sync(0xffffffffu, range, o));
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = range;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t w = 1; w < blockDim.x / 32; ++w) range = fmaxf(range, red[w]);
        const float s = affine && range > 0.f ? range / 255.f : 1.f;
        grid[0]       = affine ? 1.f : 0.f;
        grid[1]       = s;
        grid[2]       = 1.f / s;
    }
}

size_t u8_grid_ws_bytes(uint32_t D) { return sizeof(uint32_t) * (2ull * D + 1); }

cudaError_t launch_u8_grid(const float* vecs, uint64_t n, uint32_t D, void* ws, float* lo, float* grid,
                           cudaStream_t st) {
    auto*       mn  = static_cast<uint32_t*>(ws);
    uint32_t*   mx  = mn + D;
    uint32_t*   off = mx + D;
    cudaError_t e   = cudaMemsetAsync(mn, 0xff, sizeof(uint32_t) * D, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(mx, 0, sizeof(uint32_t) * (D + 1), st);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        const dim3 g((unsigned)((n + 1023) / 1024), (D + 127) / 128);
        u8_minmax_kernel<<<g, 128, 0, st>>>(vecs, n, D, mn, mx, off);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    u8_grid_kernel<<<1, 256, 0, st>>>(mn, mx, off, D, lo, grid);
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
// (parth/tools/vamana.py:25-29).  The column sums do not depend on the order in
// which blocks add them, so the medoid is the same on every run: each element is
// put on a fixed-point grid of its column, x * 2^(B - e_d), where 2^e_d bounds the
// column's magnitudes and n * 2^B < 2^63, and the terms are added as 64-bit
// integers, which is exact.  For integer-valued rows every term is exact and the
// means equal a sequential FP64 sum divided by n.  The squared distances to the
// mean are summed sequentially over d without contraction (as the oracle does).
__global__ void col_bound_kernel(const float* vecs, uint64_t n, uint32_t D, uint32_t* bound) {
    const uint32_t d = threadIdx.x + blockIdx.y * blockDim.x;
    if (d >= D) return;
    const uint64_t r0 = blockIdx.x * (uint64_t)1024;
    const uint64_t r1 = n < r0 + 1024 ? n : r0 + 1024;
    uint32_t       m  = 0u;
    for (uint64_t r = r0; r < r1; ++r) m = max(m, __float_as_uint(fabsf(vecs[r * D + d])));
    atomicMax(bound + d, m);
}
__global__ void col_sum_kernel(const float* vecs, uint64_t n, uint32_t D, const uint32_t* bound, int B,
                               unsigned long long* sum) {
    const uint32_t d = threadIdx.x + blockIdx.y * blockDim.x;
    if (d >= D) return;
    const int      sh = B - column_exponent(bound[d]);
    const uint64_t r0 = blockIdx.x * (uint64_t)1024;
    const uint64_t r1 = n < r0 + 1024 ? n : r0 + 1024;
    long long      s  = 0;
    for (uint64_t r = r0; r < r1; ++r) s += llrint(ldexp((double)vecs[r * D + d], sh));
    atomicAdd(sum + d, (unsigned long long)s);
}
// in place: the integer column sums become FP64 means
__global__ void col_mean_kernel(uint64_t n, uint32_t D, const uint32_t* bound, int B, unsigned long long* sum) {
    const uint32_t d = threadIdx.x + blockIdx.x * blockDim.x;
    if (d >= D) return;
    const long long s = (long long)sum[d];
    reinterpret_cast<double*>(sum)[d] = ldexp((double)s, column_exponent(bound[d]) - B) / (double)n;
}
__global__ void medoid_dist_kernel(const float* vecs, uint64_t n, uint32_t D, const double* mean,
                                   unsigned long long* best, int pass) {
    uint64_t r = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (r >= n) return;
    double s = 0.0;
    for (uint32_t d = 0; d < D; ++d) {
        const double t = (double)vecs[r * D + d] - mean[d];
        s              = __dadd_rn(s, __dmul_rn(t, t));
    }
    unsigned long long bits = (unsigned long long)__double_as_longlong(s);
    if (pass == 0)
        atomicMin(best, bits);
    else if (bits == best[0])
        atomicMin(best + 1, (unsigned long long)r);
}
__global__ void medoid_result_kernel(const unsigned long long* best, uint32_t* out) { *out = (uint32_t)best[1]; }

static size_t align16(size_t b) { return (b + 15) & ~size_t(15); }
size_t medoid_ws_bytes(uint32_t D) { return align16(sizeof(double) * D) + align16(sizeof(uint32_t) * D) + 16; }
unsigned long long* medoid_best(void* ws, uint32_t D) {
    return reinterpret_cast<unsigned long long*>(static_cast<char*>(ws) + align16(sizeof(double) * D) +
                                                 align16(sizeof(uint32_t) * D));
}
cudaError_t launch_col_bounds(const float* vecs, uint64_t n, uint32_t D, uint32_t* bound, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(bound, 0, sizeof(uint32_t) * D, st);
    if (e != cudaSuccess || n == 0) return e;
    const dim3 g((unsigned)((n + 1023) / 1024), (D + 127) / 128);
    col_bound_kernel<<<g, 128, 0, st>>>(vecs, n, D, bound);
    return cudaGetLastError();
}

static cudaError_t launch_col_means_f64(const float* vecs, uint64_t n, uint32_t D, void* ws, cudaStream_t st) {
    auto* sum   = static_cast<unsigned long long*>(ws);
    auto* bound = reinterpret_cast<uint32_t*>(static_cast<char*>(ws) + align16(sizeof(double) * D));
    int   lg    = 1;  // ceil(log2(n)), at least 1
    while (lg < 63 && (1ull << lg) < n) ++lg;
    const int   B = 62 - lg;
    cudaError_t e = cudaMemsetAsync(ws, 0, align16(sizeof(double) * D) + align16(sizeof(uint32_t) * D), st);
    if (e != cudaSuccess) return e;
    const dim3 g((unsigned)((n + 1023) / 1024), (D + 127) / 128);
    col_bound_kernel<<<g, 128, 0, st>>>(vecs, n, D, bound);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    col_sum_kernel<<<g, 128, 0, st>>>(vecs, n, D, bound, B, sum);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    col_mean_kernel<<<(D + 127) / 128, 128, 0, st>>>(n, D, bound, B, sum);
    return cudaGetLastError();
}

__global__ void f64_to_f32_kernel(const double* in, uint32_t n, float* out) {
    const uint32_t i = threadIdx.x + blockIdx.x * blockDim.x;
    if (i < n) out[i] = (float)in[i];
}

cudaError_t launch_col_mean(const float* vecs, uint64_t n, uint32_t D, void* ws, float* mean, cudaStream_t st) {
    if (n == 0 || D == 0) return cudaErrorInvalidValue;
    cudaError_t e = launch_col_means_f64(vecs, n, D, ws, st);
    if (e != cudaSuccess) return e;
    f64_to_f32_kernel<<<(D + 127) / 128, 128, 0, st>>>(static_cast<const double*>(ws), D, mean);
    return cudaGetLastError();
}

cudaError_t launch_medoid(const float* vecs, uint64_t n, uint32_t D, void* ws, uint32_t* d_out, cudaStream_t st) {
    if (n == 0 || D == 0) return cudaErrorInvalidValue;
    unsigned long long* best = medoid_best(ws, D);
    cudaError_t         e    = launch_col_means_f64(vecs, n, D, ws, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(best, 0xff, 2 * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const double* mean = static_cast<const double*>(ws);
    for (int pass = 0; pass < 2; ++pass) {
        medoid_dist_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(vecs, n, D, mean, best, pass);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (d_out != nullptr) {
        medoid_result_kernel<<<1, 1, 0, st>>>(best, d_out);
        e = cudaGetLastError();
    }
    return e;
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

// FreshDiskANN consolidation candidates (Algorithm 4): for each live node p with a
// deleted out-neighbour, p's live out-neighbours in order, each deleted one
// replaced in place by its own live out-neighbours; p itself, deleted ids and
// repeats are skipped, and the list stops at `cap`.  One warp per node: runs of
// live neighbours and each deleted neighbour's list go in as chunks of up to 32;
// repeats inside a chunk fall to __match_any_sync, repeats of earlier chunks to a
// hash set in shared memory (open addressing).  Distances are left to RobustPrune,
// which computes them exactly.
__global__ void consolidate_candidates_kernel(const uint32_t* deg, const uint32_t* adj, uint32_t R,
                                              const uint32_t* tomb, uint64_t first, uint64_t n,
                                              uint32_t* node_list, uint32_t* n_list, uint32_t* cand,
                                              uint32_t* cand_n, uint32_t cap, uint32_t hbits) {
    extern __shared__ uint32_t table_all[];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t hs   = 1u << hbits;
    uint32_t*      tab  = table_all + (threadIdx.x >> 5) * hs;
    auto dead = [&](uint32_t id) { return (__ldg(tomb + (id >> 5)) >> (id & 31u)) & 1u; };
    for (uint64_t p = first + blockIdx.x * (uint64_t)(blockDim.x / 32) + (threadIdx.x >> 5); p < first + n;
         p += (uint64_t)gridDim.x * (blockDim.x / 32)) {
        if (dead((uint32_t)p)) continue;
        const uint32_t dg = min(deg[p], R);
        uint32_t       v  = lane < dg ? adj[p * R + lane] : kNone;
        uint32_t       v2 = lane + 32u < dg ? adj[p * R + 32u + lane] : kNone;
        const bool     d1 = v != kNone && dead(v), d2 = v2 != kNone && dead(v2);
        uint32_t       dm = __ballot_sync(0xffffffffu, d1), dm2 = __ballot_sync(0xffffffffu, d2);
        bool           any = dm != 0u || dm2 != 0u;
        for (uint32_t j = 64; !any && j < dg; j += 32) {  // R > 64
            const uint32_t w = j + lane < dg ? adj[p * R + j + lane] : kNone;
            any              = __ballot_sync(0xffffffffu, w != kNone && dead(w)) != 0u;
        }
        if (!any) continue;
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(n_list, 1u);
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (lane == 0) node_list[slot] = (uint32_t)p;
        for (uint32_t i = lane; i < hs; i += 32) tab[i] = kNone;
        __syncwarp();
        uint32_t* c   = cand + (uint64_t)slot * cap;
        uint32_t  cnt = 0;
        // one chunk: lane's id u when `valid`, appended in lane order unless seen
        auto push = [&](uint32_t u, bool valid) {
            const bool     ok    = valid && u != (uint32_t)p && !dead(u);
            const uint32_t oks   = __ballot_sync(0xffffffffu, ok);
            const uint32_t peers = __match_any_sync(0xffffffffu, ok ? u : kNone) & oks;
            bool           fresh = false;
            if (ok && (__ffs(peers) - 1u) == lane) {  // first lane holding u
                uint32_t h = (u * 2654435761u) >> (32u - hbits);
                for (uint32_t probe = 0; probe < hs; ++probe, h = (h + 1u) & (hs - 1u)) {
                    const uint32_t old = atomicCAS(tab + h, kNone, u);
                    if (old == kNone) {
                        fresh = true;
                        break;
                    }
                    if (old == u) break;
                }
            }
            const uint32_t m   = __ballot_sync(0xffffffffu, fresh);
            const uint32_t pos = cnt + __popc(m & ((1u << lane) - 1u));
            if (fresh && pos < cap) c[pos] = u;
            cnt = min(cap, cnt + __popc(m));
            __syncwarp();
        };
        // the node's list in order, 32 entries at a time
        for (uint32_t j0 = 0; j0 < dg && cnt < cap; j0 += 32) {
            const uint32_t vv = j0 == 0 ? v : (j0 == 32 ? v2 : (j0 + lane < dg ? adj[p * R + j0 + lane] : kNone));
            const bool     in = j0 + lane < dg;
            uint32_t       deadm = j0 == 0 ? dm : (j0 == 32 ? dm2 : __ballot_sync(0xffffffffu, in && dead(vv)));
            uint32_t       done  = 0;  // lanes of this chunk already handled
            while (cnt < cap) {
                const uint32_t rest = deadm & ~done;
                const uint32_t d0   = rest ? __ffs(rest) - 1u : 32u;  // next deleted neighbour
                const uint32_t run  = (d0 == 32u ? ~0u : ((1u << d0) - 1u)) & ~done;
                push(vv, in && ((run >> lane) & 1u) && !((deadm >> lane) & 1u));
                if (d0 == 32u) break;
                done |= run | (1u << d0);
                const uint32_t w  = __shfl_sync(0xffffffffu, vv, d0);
                const uint32_t dw = min(deg[w], R);
                for (uint32_t k0 = 0; k0 < dw && cnt < cap; k0 += 32) {
                    const bool kin = k0 + lane < dw;
                    push(kin ? adj[(uint64_t)w * R + k0 + lane] : kNone, kin);
                }
            }
        }
        if (lane == 0) cand_n[slot] = cnt;
        __syncwarp();
    }
}
cudaError_t launch_consolidate_candidates(const uint32_t* deg, const uint32_t* adj, uint32_t R,
                                          const uint32_t* tomb, uint64_t first, uint64_t n, uint32_t* node_list,
                                          uint32_t* n_list, uint32_t* cand, uint32_t* cand_n, uint32_t cap,
                                          int num_sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    uint32_t hbits = 5;
    while ((1u << hbits) < 2u * cap) ++hbits;  // load factor <= 1/2
    const int    warps = 4;
    const size_t smem  = sizeof(uint32_t) * warps * (1u << hbits);
    cudaError_t  e = cudaFuncSetAttribute(consolidate_candidates_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e          = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, consolidate_candidates_kernel, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * num_sms;
    const uint64_t need = (n + warps - 1) / warps;
    if (grid > need) grid = need;
    consolidate_candidates_kernel<<<(unsigned)grid, warps * 32, smem, st>>>(deg, adj, R, tomb, first, n,
                                                                            node_list, n_list, cand, cand_n, cap,
                                                                            hbits);
    return cudaGetLastError();
}

}  // namespace vann

// ---------------------------------------------------------------- allocation-free medoid
// Entry-point selection (the medoid above) for callers that must not allocate
// device memory.  Its scratch -- per column a 64-bit sum (then the mean) and a
// magnitude bound, and the argmin word pair -- lives in this file-scope device
// array instead of memory the library would cudaMalloc: up to kNoAllocMaxDim
// dimensions, 48 KiB + 256 B, held by every device that loads the library until
// the process exits.
namespace {
constexpr uint32_t kNoAllocMaxDim = 4096;
constexpr size_t   kNoAllocBytes  = 12 * (size_t)kNoAllocMaxDim + 256;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// The device address of g_noalloc_scratch, resolved once per device and context:
// in host code the symbol is only a stand-in.  A context created after a
// cudaDeviceReset has its own copy of the array, so the address is resolved again
// when the current context's id changes.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
std::mutex         g_noalloc_mu;
void*              g_noalloc_addr[256] = {};
unsigned long long g_noalloc_ctx[256]  = {};
CtxGetCurrentFn    g_ctx_current       = nullptr;
CtxGetIdFn         g_ctx_id            = nullptr;
bool               g_ctx_fns_looked_up = false;

// id of the current context, 0 when it cannot be told (the address is then resolved on every call)
unsigned long long current_context_id() {
    if (!g_ctx_fns_looked_up) {
        g_ctx_fns_looked_up = true;
        void* f1 = nullptr;
        void* f2 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault) == cudaSuccess && f1 && f2) {
            g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f1);
            g_ctx_id      = reinterpret_cast<CtxGetIdFn>(f2);
        }
        (void)cudaGetLastError();  // a failed lookup leaves no error behind for the caller
    }
    if (!g_ctx_current || !g_ctx_id) return 0;
    void*              ctx = nullptr;
    unsigned long long id  = 0;
    if (g_ctx_current(&ctx) != 0 || ctx == nullptr || g_ctx_id(ctx, &id) != 0) return 0;
    return id;
}
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
    // an error left pending by earlier work is the caller's: report it as such,
    // without consuming it, so the launch check below sees only this call's launches
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        vann::set_last_error((std::string("vann_medoid_noalloc: a CUDA error was already pending: ") +
                              cudaGetErrorString(pending)).c_str());
        return VANN_ERR_CUDA;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) {
        vann::set_last_error("vann_medoid_noalloc: no current CUDA device");
        return VANN_ERR_CUDA;
    }
    void* base = nullptr;
    {
        // set-up on the first call on this device (with the device current), and
        // again in a new context: the kernels need the array's device address
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        const unsigned long long ctx = current_context_id();
        if (g_noalloc_addr[dev] == nullptr || ctx == 0 || ctx != g_noalloc_ctx[dev]) {
            void*             p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || p == nullptr) {
                vann::set_last_error((std::string("vann_medoid_noalloc: cudaGetSymbolAddress failed: ") +
                                      cudaGetErrorString(e)).c_str());
                return VANN_ERR_CUDA;
            }
            g_noalloc_addr[dev] = p;
            g_noalloc_ctx[dev]  = ctx ? ctx : current_context_id();
        }
        base = g_noalloc_addr[dev];
    }
    static_assert(12 * (size_t)kNoAllocMaxDim + 32 <= kNoAllocBytes, "scratch holds the medoid workspace");
    // launch_medoid clears the sums, bounds and argmin pair the previous call left
    const cudaError_t e =
        vann::launch_medoid(d_vecs, n, dim, base, d_medoid_out, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        vann::set_last_error((std::string("vann_medoid_noalloc: ") + cudaGetErrorString(e)).c_str());
        return VANN_ERR_CUDA;
    }
    return VANN_OK;
}

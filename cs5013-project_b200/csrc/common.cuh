// common.cuh -- device helpers shared by the search and prune kernels.
//
// Data layout in HBM (one index):
//   vecs_f32  [capacity x D]  FP32 rows, 16-byte aligned (D % 4 == 0)
//   vecs_bf16 [capacity x D]  optional traversal copy
//   vecs_fp8  [capacity x D]  optional e4m3 copy + scale_fp8[capacity]
//   vecs_u8   [capacity x D]  optional uint8 copy
//   deg       [capacity]      u32 out-degree
//   adj       [capacity x R]  u32 neighbour ids (row stride R)
//   tomb      [capacity/32]   u32 tombstone bitmap
// A warp reads one vector as 32 lanes x 4 elements (one 16/8/4-byte load per
// lane per 128 dimensions), so every row gather is a single coalesced request.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace vann {

constexpr uint32_t kBloomSlots = 39988u;                 // bloom_filter.cuh:7
constexpr uint32_t kBloomWords = (kBloomSlots + 31) / 32;  // bit-packed, 5000 B
constexpr uint32_t kVisitedBit = 0x80000000u;            // worklist id flag
constexpr uint32_t kNone       = 0xFFFFFFFFu;

// status word bits (device side)
constexpr uint32_t kStatusHopLimit = 1u;
constexpr uint32_t kStatusOverflow = 2u;

// ---------------------------------------------------------------- bloom hashes
// Same functions as the reference filter (vamana/include/bloom_filter.cuh:11-30):
// byte-wise FNV-style folding in 64-bit arithmetic, modulo 39,988.  They must be
// identical for the filter's false positives to steer searches the same way.
__device__ __forceinline__ uint32_t bloom_h1(uint32_t x) {
    uint64_t h = 0xcbf29ce4ull;
    h          = (h ^ (x & 0xffu)) * 0x01000193ull;
    h          = (h ^ ((x >> 8) & 0xffu)) * 0x01000193ull;
    h          = (h ^ ((x >> 16) & 0xffu)) * 0x01000193ull;
    h          = (h ^ ((x >> 24) & 0xffu)) * 0x01000193ull;
    return (uint32_t)(h % kBloomSlots);
}
__device__ __forceinline__ uint32_t bloom_h2(uint32_t x) {
    uint64_t h = 0x84222325ull;
    h          = (h ^ (x & 0xffu)) * 0x1B3ull;
    h          = (h ^ ((x >> 8) & 0xffu)) * 0x1B3ull;
    h          = (h ^ ((x >> 16) & 0xffu)) * 0x1B3ull;
    h          = (h ^ ((x >> 24) & 0xffu)) * 0x1B3ull;
    return (uint32_t)(h % kBloomSlots);
}

// ---------------------------------------------------------------- stores
struct StoreF32 {
    static constexpr int kBytes = 4;
    __device__ __forceinline__ static float4 load4(const void* base, const float*, uint64_t row,
                                                   uint32_t D, uint32_t c) {
        const float4* p = reinterpret_cast<const float4*>(static_cast<const float*>(base) + row * D);
        return __ldg(p + c);
    }
};
struct StoreBF16 {
    static constexpr int kBytes = 2;
    __device__ __forceinline__ static float4 load4(const void* base, const float*, uint64_t row,
                                                   uint32_t D, uint32_t c) {
        const uint2* p =
            reinterpret_cast<const uint2*>(static_cast<const __nv_bfloat16*>(base) + row * D);
        uint2 u = __ldg(p + c);
        float4 r;
        r.x = __uint_as_float(u.x << 16);
        r.y = __uint_as_float(u.x & 0xffff0000u);
        r.z = __uint_as_float(u.y << 16);
        r.w = __uint_as_float(u.y & 0xffff0000u);
        return r;
    }
};
struct StoreFP8 {
    static constexpr int kBytes = 1;
    __device__ __forceinline__ static float4 load4(const void* base, const float* scale,
                                                   uint64_t row, uint32_t D, uint32_t c) {
        const uint32_t* p =
            reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(base) + row * D);
        uint32_t u = __ldg(p + c);
        float    s = __ldg(scale + row);
        __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(u & 0xffffu), __NV_E4M3);
        __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(u >> 16), __NV_E4M3);
        float2 a = __half22float2(*reinterpret_cast<__half2*>(&lo));
        float2 b = __half22float2(*reinterpret_cast<__half2*>(&hi));
        return make_float4(a.x * s, a.y * s, b.x * s, b.y * s);
    }
};
struct StoreU8 {
    static constexpr int kBytes = 1;
    __device__ __forceinline__ static float4 load4(const void* base, const float*, uint64_t row,
                                                   uint32_t D, uint32_t c) {
        const uint32_t* p =
            reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(base) + row * D);
        uint32_t u = __ldg(p + c);
        return make_float4((float)(u & 0xffu), (float)((u >> 8) & 0xffu), (float)((u >> 16) & 0xffu),
                           (float)(u >> 24));
    }
};

__device__ __forceinline__ float sqdiff4(const float4& q, const float4& x, float acc) {
    float d0 = q.x - x.x, d1 = q.y - x.y, d2 = q.z - x.z, d3 = q.w - x.w;
    acc      = fmaf(d0, d0, acc);
    acc      = fmaf(d1, d1, acc);
    acc      = fmaf(d2, d2, acc);
    acc      = fmaf(d3, d3, acc);
    return acc;
}

// Reduce 8 per-lane partial sums across the warp in 9 shuffles.  On return the
// lane holds the full sum of value index vidx(lane) =
// ((lane>>4)&1)*4 + ((lane>>3)&1)*2 + ((lane>>2)&1); the sum of value j is held
// by lane vlane(j) = ((j>>2)&1)*16 + ((j>>1)&1)*8 + (j&1)*4.
__device__ __forceinline__ float transpose_reduce8(const float v[8], uint32_t lane) {
    float w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        bool  up   = lane & 16;
        float send = up ? v[i] : v[i + 4];
        float keep = up ? v[i + 4] : v[i];
        w[i]       = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    float x[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        bool  up   = lane & 8;
        float send = up ? w[i] : w[i + 2];
        float keep = up ? w[i + 2] : w[i];
        x[i]       = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    bool  up   = lane & 4;
    float send = up ? x[0] : x[1];
    float keep = up ? x[1] : x[0];
    float y    = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    y += __shfl_xor_sync(0xffffffffu, y, 2);
    y += __shfl_xor_sync(0xffffffffu, y, 1);
    return y;
}
__device__ __forceinline__ uint32_t vidx_of_lane(uint32_t lane) {
    return ((lane >> 4) & 1u) * 4u + ((lane >> 3) & 1u) * 2u + ((lane >> 2) & 1u);
}
__device__ __forceinline__ uint32_t lane_of_vidx(uint32_t j) {
    return ((j >> 2) & 1u) * 16u + ((j >> 1) & 1u) * 8u + (j & 1u) * 4u;
}

// Squared L2 from the warp's register-resident query chunks to up to 8 rows.
// ids[j] for j < cnt (uniform across the warp).  Returns, in lane vlane(j),
// the distance to row j.  All loads are issued before the arithmetic.
template <typename S, int NCH>
__device__ __forceinline__ float dist8(const float4 (&q)[NCH], const void* base, const float* scale,
                                       const uint32_t (&ids)[8], int cnt, uint32_t D,
                                       uint32_t lane) {
    const uint32_t nchunk = D >> 2;
    float4         x[8][NCH];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            uint32_t ch = lane + 32u * c;
            if (j < cnt && ch < nchunk)
                x[j][c] = S::load4(base, scale, ids[j], D, ch);
            else
                x[j][c] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
    }
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            uint32_t ch = lane + 32u * c;
            if (j < cnt && ch < nchunk) acc = sqdiff4(q[c], x[j][c], acc);
        }
        v[j] = acc;
    }
    return transpose_reduce8(v, lane);
}

template <int NCH>
__device__ __forceinline__ void load_query_f32(float4 (&q)[NCH], const float* row, uint32_t D,
                                               uint32_t lane) {
    const uint32_t nchunk = D >> 2;
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
        uint32_t ch = lane + 32u * c;
        q[c] = ch < nchunk ? __ldg(reinterpret_cast<const float4*>(row) + ch)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// ---------------------------------------------------------------- keys
// Non-negative float distances order like their bit patterns.
__device__ __forceinline__ uint64_t make_key(float d, uint32_t lo) {
    return ((uint64_t)__float_as_uint(d) << 32) | lo;
}
__device__ __forceinline__ float key_dist(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }

// Warp bitonic sort of SPL*32 keys held as key[s] = element s*32 + lane.
template <int SPL>
__device__ __forceinline__ void warp_bitonic_sort(uint64_t (&key)[SPL], uint32_t lane) {
    constexpr int N = SPL * 32;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int js = j / 32;
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    int p = s ^ js;
                    if (p > s) {
                        uint32_t e   = (uint32_t)s * 32u + lane;
                        bool     asc = (e & (uint32_t)k) == 0;
                        uint64_t a = key[s], b = key[p];
                        bool     sw = asc ? (a > b) : (a < b);
                        if (sw) {
                            key[s] = b;
                            key[p] = a;
                        }
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    uint32_t e     = (uint32_t)s * 32u + lane;
                    uint64_t other = __shfl_xor_sync(0xffffffffu, key[s], j);
                    bool     asc   = (e & (uint32_t)k) == 0;
                    bool     lower = (lane & (uint32_t)j) == 0;
                    uint64_t mn = key[s] < other ? key[s] : other;
                    uint64_t mx = key[s] < other ? other : key[s];
                    key[s]      = (asc == lower) ? mn : mx;
                }
            }
        }
    }
}

// Warp bitonic sort of n (power of two, >= 32) keys in shared memory.
__device__ __forceinline__ void warp_bitonic_sort_smem(uint64_t* key, uint32_t n, uint32_t lane) {
    for (uint32_t k = 2; k <= n; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t e = lane; e < n; e += 32) {
                uint32_t p = e ^ j;
                if (p > e) {
                    bool     asc = (e & k) == 0;
                    uint64_t a = key[e], b = key[p];
                    if (asc ? (a > b) : (a < b)) {
                        key[e] = b;
                        key[p] = a;
                    }
                }
            }
            __syncwarp();
        }
    }
}

}  // namespace vann

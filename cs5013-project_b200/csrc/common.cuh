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

// Both filter slots of one id packed as (h1 << 16) | h2 (each < 39,988 < 2^16).
// The index keeps this word beside every adjacency entry, so a search reads the
// slots of a parent's neighbours in the same request as their ids.
__device__ __forceinline__ uint32_t bloom_pack(uint32_t x) { return (bloom_h1(x) << 16) | bloom_h2(x); }

// ---------------------------------------------------------------- stores
// Each store reads one 4-element chunk of a row per lane (16, 8 or 4 bytes), so
// a warp reads a whole 128-dim row in one coalesced request.  kGroup rows are
// gathered per round (32 registers of raw data per lane whatever the width):
// narrower elements mean fewer dependent gather rounds per expansion.
struct StoreF32 {
    static constexpr int  kGroup  = 8;
    static constexpr bool kScaled = false;
    static constexpr bool kBytes8 = false;
    using raw_t                   = float4;
    __device__ __forceinline__ static raw_t load(const void* base, uint64_t row, uint32_t D, uint32_t c) {
        return __ldg(reinterpret_cast<const float4*>(static_cast<const float*>(base) + row * D) + c);
    }
    __device__ __forceinline__ static raw_t zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
    __device__ __forceinline__ static float4 widen(const raw_t& x, float) { return x; }
};
struct StoreBF16 {
    static constexpr int  kGroup  = 16;
    static constexpr bool kScaled = false;
    static constexpr bool kBytes8 = false;
    using raw_t                   = uint2;
    __device__ __forceinline__ static raw_t load(const void* base, uint64_t row, uint32_t D, uint32_t c) {
        return __ldg(reinterpret_cast<const uint2*>(static_cast<const __nv_bfloat16*>(base) + row * D) + c);
    }
    __device__ __forceinline__ static raw_t zero() { return make_uint2(0u, 0u); }
    __device__ __forceinline__ static float4 widen(const raw_t& u, float) {
        return make_float4(__uint_as_float(u.x << 16), __uint_as_float(u.x & 0xffff0000u),
                           __uint_as_float(u.y << 16), __uint_as_float(u.y & 0xffff0000u));
    }
};
struct StoreFP8 {
    static constexpr int  kGroup  = 16;
    static constexpr bool kScaled = true;
    static constexpr bool kBytes8 = false;
    using raw_t                   = uint32_t;
    __device__ __forceinline__ static raw_t load(const void* base, uint64_t row, uint32_t D, uint32_t c) {
        return __ldg(reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(base) + row * D) + c);
    }
    __device__ __forceinline__ static raw_t zero() { return 0u; }
    __device__ __forceinline__ static float4 widen(const raw_t& u, float s) {
        __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(u & 0xffffu), __NV_E4M3);
        __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(u >> 16), __NV_E4M3);
        float2 a = __half22float2(*reinterpret_cast<__half2*>(&lo));
        float2 b = __half22float2(*reinterpret_cast<__half2*>(&hi));
        return make_float4(a.x * s, a.y * s, b.x * s, b.y * s);
    }
};
struct StoreU8 {
    static constexpr int  kGroup  = 32;
    static constexpr bool kScaled = false;
    static constexpr bool kBytes8 = true;  // exact integer path for integer queries
    using raw_t                   = uint32_t;
    __device__ __forceinline__ static raw_t load(const void* base, uint64_t row, uint32_t D, uint32_t c) {
        return __ldg(reinterpret_cast<const uint32_t*>(static_cast<const uint8_t*>(base) + row * D) + c);
    }
    __device__ __forceinline__ static raw_t zero() { return 0u; }
    __device__ __forceinline__ static float4 widen(const raw_t& u, float) {
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

// Register-resident query: FP32 chunks, plus packed uint8 chunks and |q|^2 when
// every element is an integer in [0, 255] (then uint8 rows use dp4a exactly).
template <int NCH>
struct Query {
    float4   f[NCH];
    uint32_t u[NCH];
    int      qq;
    bool     qint;
};

template <int NCH>
__device__ __forceinline__ void load_query(Query<NCH>& q, const float* row, uint32_t D, uint32_t lane) {
    const uint32_t nchunk = D >> 2;
    bool           ok     = true;
    int            qq     = 0;
#pragma unroll
    for (int c = 0; c < NCH; ++c) {
        uint32_t ch = lane + 32u * c;
        float4   v  = ch < nchunk ? __ldg(reinterpret_cast<const float4*>(row) + ch)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
        q.f[c]      = v;
        float e[4]  = {v.x, v.y, v.z, v.w};
        uint32_t pk = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            bool good = e[i] >= 0.f && e[i] <= 255.f && rintf(e[i]) == e[i];
            ok &= good;
            uint32_t b = good ? (uint32_t)e[i] : 0u;
            pk |= b << (8 * i);
            qq += (int)(b * b);
        }
        q.u[c] = pk;
    }
    q.qint = __all_sync(0xffffffffu, ok);
#pragma unroll
    for (int o = 16; o; o >>= 1) qq += __shfl_xor_sync(0xffffffffu, qq, o);
    q.qq = qq;
}

// Reduce G per-lane partial sums across the warp with log2(G) exchange levels
// plus 5 - log2(G) butterfly levels (31 shuffles for G = 32, 9 for G = 8).  On
// return lane l holds the full sum of value l >> (5 - log2 G).
template <int G, typename T>
__device__ __forceinline__ T transpose_reduce(T (&v)[G], uint32_t lane) {
    constexpr int LOG2G = G == 32 ? 5 : G == 16 ? 4 : G == 8 ? 3 : G == 4 ? 2 : G == 2 ? 1 : 0;
    static_assert((1 << LOG2G) == G, "G must be a power of two <= 32");
#pragma unroll
    for (int lvl = 0; lvl < LOG2G; ++lvl) {
        const int  half = G >> (lvl + 1);
        const int  off  = 16 >> lvl;
        const bool up   = (lane & (uint32_t)off) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            T send = up ? v[i] : v[i + half];
            T keep = up ? v[i + half] : v[i];
            v[i]   = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    T y = v[0];
#pragma unroll
    for (int off = 16 >> LOG2G; off >= 1; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
    return y;
}
template <int G>
__device__ __forceinline__ uint32_t group_slot_of_lane(uint32_t lane) {
    constexpr int LOG2G = G == 32 ? 5 : G == 16 ? 4 : G == 8 ? 3 : 0;
    return lane >> (5 - LOG2G);
}
template <int G>
__device__ __forceinline__ bool group_writer(uint32_t lane) {
    constexpr int LOG2G = G == 32 ? 5 : G == 16 ? 4 : G == 8 ? 3 : 0;
    return (lane & ((1u << (5 - LOG2G)) - 1u)) == 0u;
}

// Squared L2 from the query to up to S::kGroup rows ids[0..cnt) (ids in shared
// memory, cnt uniform across the warp).  Every row's loads are issued before
// any arithmetic.  Returns, in lane l, the distance to row group_slot_of_lane(l).
template <typename S, int NCH, typename IdFn>
__device__ __forceinline__ float dist_group(const Query<NCH>& q, const void* base, const float* scale,
                                            IdFn ids, int cnt, uint32_t D, uint32_t lane) {
    constexpr int  G      = S::kGroup;
    const uint32_t nchunk = D >> 2;
    typename S::raw_t x[G][NCH];
    float             sc[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
        uint32_t id = j < cnt ? ids(j) : 0u;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            uint32_t ch = lane + 32u * c;
            x[j][c]     = (j < cnt && ch < nchunk) ? S::load(base, id, D, ch) : S::zero();
        }
        if constexpr (S::kScaled) sc[j] = j < cnt ? __ldg(scale + id) : 0.f;
        else sc[j] = 1.f;
    }
    if constexpr (S::kBytes8) {
        if (q.qint) {
            int v[G];
#pragma unroll
            for (int j = 0; j < G; ++j) {
                int acc = 0;
#pragma unroll
                for (int c = 0; c < NCH; ++c) {
                    int xx = __dp4a((unsigned)x[j][c], (unsigned)x[j][c], 0u);
                    int qx = __dp4a((unsigned)q.u[c], (unsigned)x[j][c], 0u);
                    acc += xx - 2 * qx;
                }
                v[j] = acc;
            }
            int y = transpose_reduce<G, int>(v, lane);
            return (float)(y + q.qq);
        }
    }
    float v[G];
#pragma unroll
    for (int j = 0; j < G; ++j) {
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            uint32_t ch = lane + 32u * c;
            if (ch < nchunk) acc = sqdiff4(q.f[c], S::widen(x[j][c], sc[j]), acc);
        }
        v[j] = acc;
    }
    return transpose_reduce<G, float>(v, lane);
}

// ---------------------------------------------------------------- keys
// Non-negative float distances order like their bit patterns.
__device__ __forceinline__ uint64_t make_key(float d, uint32_t lo) {
    return ((uint64_t)__float_as_uint(d) << 32) | lo;
}
__device__ __forceinline__ float key_dist(uint64_t k) { return __uint_as_float((uint32_t)(k >> 32)); }

// Warp bitonic sort of the first n (power of two <= SPL*32) keys held as
// key[s] = element s*32 + lane; elements at or beyond n are not touched.
template <int SPL>
__device__ __forceinline__ void warp_bitonic_sort(uint64_t (&key)[SPL], uint32_t lane,
                                                  uint32_t n = SPL * 32) {
    constexpr int N = SPL * 32;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
        if ((uint32_t)k > n) break;
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

// common.cuh -- device helpers shared by the search and prune kernels.
//
// Data layout in HBM (one index):
//   vecs_f32  [capacity x D]  FP32 rows, 16-byte aligned (D % 4 == 0)
//   vecs_bf16 [capacity x D]  optional traversal copy
//   vecs_fp8  [capacity x D]  optional e4m3 copy + per row (scale, scale^2 |codes|^2)
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

#include <utility>

namespace vann {

constexpr uint32_t kBloomSlots = 39988u;                 // bloom_filter.cuh:7
constexpr uint32_t kBloomWords = (kBloomSlots + 31) / 32;  // bit-packed, 5000 B
constexpr uint32_t kVisitedBit = 0x80000000u;            // worklist id flag
constexpr uint32_t kNone       = 0xFFFFFFFFu;

// status word bits (device side)
constexpr uint32_t kStatusHopLimit = 1u;
constexpr uint32_t kStatusOverflow = 2u;
constexpr uint32_t kStatusTimeout  = 4u;  // a bounded device wait gave up

// words of the index's device status array
constexpr uint32_t kWordStatus   = 0;  // kStatus* bits, cleared by vann_sync
constexpr uint32_t kWordU8Inexact = 1;  // set when a row was not an integer in [0, 255]
constexpr uint32_t kWordPruned    = 4;  // 2 x u64: nodes pruned by prune_tc_kernel, by prune_kernel

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
// Rows are read in 16-byte chunks: 4 FP32, 8 BF16 or 16 one-byte elements.  A
// row of C chunks is spread over T = C lanes (T <= 32, CPL chunks per lane when
// C > 32), so one warp load instruction reads 32 / T whole rows, coalesced, and
// each lane reduces 16 bytes before a log2(T)-level shuffle reduction.  M rows
// per lane group are gathered per round with all loads in flight first, so a
// round covers G = M * 32 / T rows: 8 (FP32), 16 (BF16) or 32 (one-byte rows).
// Dimension class DC: D <= 128 << DC.
// widen2 / codes2 give the elements of a 16-byte chunk as pairs (element 2p in .x,
// 2p + 1 in .y) for the packed FP32 arithmetic of sm_100 (__ffma2_rn: two FMAs
// per instruction).
struct StoreF32 {
    static constexpr int  kElems = 4, kLanes128 = 32, kM = 8;
    static constexpr bool kScaled = false, kInt = false, kPQ = false;
    __device__ __forceinline__ static void widen2(const uint4& r, float2 (&o)[2]) {
        o[0] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
        o[1] = make_float2(__uint_as_float(r.z), __uint_as_float(r.w));
    }
};
struct StoreBF16 {
    static constexpr int  kElems = 8, kLanes128 = 16, kM = 8;
    static constexpr bool kScaled = false, kInt = false, kPQ = false;
    // a BF16 is the upper half of its FP32 value
    __device__ __forceinline__ static void widen2(const uint4& r, float2 (&o)[4]) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = make_float2(__uint_as_float(w[i] << 16), __uint_as_float(w[i] & 0xffff0000u));
    }
};
struct StoreFP8 {
    static constexpr int  kElems = 16, kLanes128 = 8, kM = 8;
    static constexpr bool kScaled = true, kInt = false, kPQ = false;
    // the 16 codes of a chunk, unscaled: one e4m3x2 -> f16x2 conversion per pair,
    // then f16 -> f32 (both exact)
    __device__ __forceinline__ static void codes2(const uint4& r, float2 (&o)[8]) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            __half2_raw lo = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] & 0xffffu), __NV_E4M3);
            __half2_raw hi = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)(w[i] >> 16), __NV_E4M3);
            o[2 * i]       = __half22float2(*reinterpret_cast<__half2*>(&lo));
            o[2 * i + 1]   = __half22float2(*reinterpret_cast<__half2*>(&hi));
        }
    }
};
struct StoreU8 {
    static constexpr int  kElems = 16, kLanes128 = 8, kM = 8;
    static constexpr bool kScaled = false, kInt = true, kPQ = false;  // exact dp4a path for integer queries
    __device__ __forceinline__ static void widen(const uint4& r, float (&o)[16]) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            o[4 * i]     = (float)(w[i] & 0xffu);
            o[4 * i + 1] = (float)((w[i] >> 8) & 0xffu);
            o[4 * i + 2] = (float)((w[i] >> 16) & 0xffu);
            o[4 * i + 3] = (float)(w[i] >> 24);
        }
    }
};
// Product-quantized codes (pq.cu): one byte per subspace of kPqSub = 8 dimensions,
// so a 16-byte chunk holds the codes of 128 dimensions.  A row's distance is the
// sum of its codes' entries in the query's table (one lane per 16 codes).
struct StorePQ {
    static constexpr int  kElems = 128, kLanes128 = 1, kM = 1;
    static constexpr bool kScaled = false, kInt = false, kPQ = true;
};
constexpr uint32_t kPqSub = 8;    // dimensions per subspace
constexpr uint32_t kPqK   = 256;  // centroids per subspace (one byte per code)

// Lanes per row (kT), 16-byte chunks per lane (kCPL) and rows per lane (kM) of
// store S in dimension class DC.  In the smallest dimension class, integer, FP32
// and BF16 rows give each lane two adjacent chunks (32 contiguous bytes, one
// 256-bit load) and half the rows per round: the same rows per gather round for
// half the row-id loads, addresses and cross-lane reduction levels.
template <typename S, int DC>
struct Layout {
    static constexpr int  kChunks = S::kLanes128 << DC;
    static constexpr bool kNarrow = DC == 0 && kChunks >= 8 && (S::kInt || (!S::kScaled && !S::kPQ));
    static constexpr int  kT   = kNarrow ? kChunks / 2 : (kChunks < 32 ? kChunks : 32);
    static constexpr int  kCPL = kChunks / kT;
    static constexpr int  kP   = 32 / kT;                       // rows per warp load
    static constexpr int  kM   = kNarrow ? S::kM / 2 : S::kM;   // rows per lane per round
    static constexpr int  kG   = kM * kP;                       // rows per gather round
    // chunk c of lane group member t: adjacent pairs in the narrow layout, else
    // interleaved
    __device__ __forceinline__ static uint32_t chunk(uint32_t t, int c) {
        return kNarrow ? t * (uint32_t)kCPL + (uint32_t)c : t + (uint32_t)kT * (uint32_t)c;
    }
};

__device__ __forceinline__ uint4 load16(const void* base, uint64_t row_bytes, uint64_t row, uint32_t k) {
    return __ldg(reinterpret_cast<const uint4*>(static_cast<const unsigned char*>(base) + row * row_bytes) + k);
}
// chunks k and k + 1 of a row (32 bytes, 32-byte aligned) in one 256-bit load
__device__ __forceinline__ void load32(const void* base, uint64_t row_bytes, uint64_t row, uint32_t k, uint4& a,
                                       uint4& b) {
    const unsigned char* p = static_cast<const unsigned char*>(base) + row * row_bytes + 16ull * k;
    asm("ld.global.nc.v8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
        : "l"(p));
}

// Register-resident query in the lane layout of store S: the lane's chunks in
// FP32, plus packed uint8 words and |q|^2 when every element is an integer in
// [0, 255] (uint8 rows then use exact dp4a integer arithmetic).
template <typename S, int DC>
struct Query {
    // FP32 copy of the lane's chunks as element pairs (integer stores keep none:
    // their rare non-integer fallback re-reads the row through L1)
    float2       f2[S::kInt || S::kPQ ? 1 : Layout<S, DC>::kCPL][S::kInt || S::kPQ ? 1 : S::kElems / 2];
    uint32_t     u[S::kPQ ? 1 : Layout<S, DC>::kCPL][S::kPQ ? 1 : S::kElems / 4];
    const uint16_t* lut;        // PQ: this warp's distance table [D / 8][256] in shared memory
    float           lut_scale;  // PQ: distance = scale * sum of table entries
    const float* row;
    int          qq;
    float        qn;  // this lane's share of |q|^2 (scaled stores)
    bool         qint;
};

// center (scaled stores): the per-dimension centre the row codes are relative to;
// the query is centred the same way, which leaves every distance unchanged.
template <typename S, int DC>
__device__ __forceinline__ void load_query(Query<S, DC>& q, const float* row, uint32_t D, uint32_t lane,
                                           const float* center = nullptr) {
    if constexpr (S::kPQ) {  // the PQ query is its distance table (build_pq_lut)
        q.row  = row;
        q.qint = false;
        return;
    }
    using Ly              = Layout<S, DC>;
    const uint32_t chunks = D / S::kElems;
    const uint32_t t      = lane % Ly::kT;
    bool           ok     = true;
    int            qq     = 0;
    float          qn     = 0.f;
#pragma unroll
    for (int c = 0; c < Ly::kCPL; ++c) {
        uint32_t k     = Ly::chunk(t, c);
        bool     valid = k < chunks;
#pragma unroll
        for (int v = 0; v < S::kElems / 4; ++v) {
            float4 x = valid ? __ldg(reinterpret_cast<const float4*>(row + k * S::kElems) + v)
                             : make_float4(0.f, 0.f, 0.f, 0.f);
            if constexpr (S::kScaled) {
                if (center != nullptr && valid) {
                    const float4 cz = __ldg(reinterpret_cast<const float4*>(center + k * S::kElems) + v);
                    x.x -= cz.x;
                    x.y -= cz.y;
                    x.z -= cz.z;
                    x.w -= cz.w;
                }
            }
            float  e[4] = {x.x, x.y, x.z, x.w};
            if constexpr (!S::kInt) {
                q.f2[c][2 * v]     = make_float2(x.x, x.y);
                q.f2[c][2 * v + 1] = make_float2(x.z, x.w);
            }
            uint32_t pk = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if constexpr (S::kScaled) qn = fmaf(e[i], e[i], qn);
                bool good = e[i] >= 0.f && e[i] <= 255.f && rintf(e[i]) == e[i];
                ok &= good;
                uint32_t b = good ? (uint32_t)e[i] : 0u;
                pk |= b << (8 * i);
                qq += (int)(b * b);
            }
            q.u[c][v] = pk;
        }
    }
    q.row  = row;
    q.qn   = qn;
    q.qint = __all_sync(0xffffffffu, ok);
    // each group of T lanes holds the whole query
#pragma unroll
    for (int o = Ly::kT / 2; o >= 1; o >>= 1) qq += __shfl_xor_sync(0xffffffffu, qq, o);
    q.qq = qq;
}

// The query of an integer store taken straight from a row of the exact uint8 copy
// (the caller knows every row there equals its FP32 row): the lane's chunks as
// packed words, |q|^2 from dp4a.  The same Query as load_query gives for that FP32
// row, from a quarter of the bytes and without the per-element checks.
template <typename S, int DC>
__device__ __forceinline__ void load_query_u8row(Query<S, DC>& q, const uint8_t* row, uint32_t D, uint32_t lane) {
    static_assert(S::kInt, "uint8 rows");
    using Ly                 = Layout<S, DC>;
    const uint32_t chunks    = D / S::kElems;
    const uint32_t t         = lane % Ly::kT;
    uint32_t       qq        = 0;
    uint4          w[Ly::kCPL];
    if constexpr (Ly::kNarrow) {
        const uint32_t k0 = Ly::chunk(t, 0);
        if (k0 + 1u < chunks && (D & 31u) == 0u) {
            load32(row, 0, 0, k0, w[0], w[1]);
        } else {
            w[0] = k0 < chunks ? load16(row, 0, 0, k0) : make_uint4(0u, 0u, 0u, 0u);
            w[1] = k0 + 1u < chunks ? load16(row, 0, 0, k0 + 1u) : make_uint4(0u, 0u, 0u, 0u);
        }
    } else {
#pragma unroll
        for (int c = 0; c < Ly::kCPL; ++c) {
            const uint32_t k = Ly::chunk(t, c);
            w[c]             = k < chunks ? load16(row, 0, 0, k) : make_uint4(0u, 0u, 0u, 0u);
        }
    }
#pragma unroll
    for (int c = 0; c < Ly::kCPL; ++c) {
        const uint32_t v[4] = {w[c].x, w[c].y, w[c].z, w[c].w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            q.u[c][i] = v[i];
            qq        = __dp4a(v[i], v[i], qq);
        }
    }
    int s = (int)qq;
#pragma unroll
    for (int o = Ly::kT / 2; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    q.qq   = s;
    q.qn   = 0.f;
    q.row  = nullptr;
    q.qint = true;
}

__device__ __forceinline__ float sqdiff(float q, float x, float acc) {
    float d = q - x;
    return fmaf(d, d, acc);
}

// Reduce M per-lane values across the T lanes of each lane group: log2(M)
// exchange levels then butterfly levels.  Lane t of a group ends with the sum
// of value t / (T / M).
template <int M, int T, typename V>
__device__ __forceinline__ V group_reduce(V (&v)[M], uint32_t lane) {
    constexpr int LOG2M = M == 32 ? 5 : M == 16 ? 4 : M == 8 ? 3 : M == 4 ? 2 : M == 2 ? 1 : 0;
    static_assert((1 << LOG2M) == M && M <= T, "M must be a power of two <= T");
#pragma unroll
    for (int lvl = 0; lvl < LOG2M; ++lvl) {
        const int  half = M >> (lvl + 1);
        const int  off  = (T / 2) >> lvl;
        const bool up   = (lane & (uint32_t)off) != 0;
#pragma unroll
        for (int i = 0; i < half; ++i) {
            V send = up ? v[i] : v[i + half];
            V keep = up ? v[i + half] : v[i];
            v[i]   = keep + __shfl_xor_sync(0xffffffffu, send, off);
        }
    }
    V y = v[0];
#pragma unroll
    for (int off = (T / 2) >> LOG2M; off >= 1; off >>= 1) y += __shfl_xor_sync(0xffffffffu, y, off);
    return y;
}

// Row (within a gather round) whose distance lane `lane` holds after dist_group,
// and whether this lane is the one that writes it.
template <typename S, int DC>
__device__ __forceinline__ uint32_t round_row_of_lane(uint32_t lane) {
    using Ly        = Layout<S, DC>;
    const uint32_t t = lane % Ly::kT, g = lane / Ly::kT;
    return (t / (Ly::kT / Ly::kM)) * Ly::kP + g;
}
template <typename S, int DC>
__device__ __forceinline__ bool round_writer(uint32_t lane) {
    using Ly = Layout<S, DC>;
    return (lane % (Ly::kT / Ly::kM)) == 0u;
}

// Squared L2 from the query to rows ids(0) .. ids(cnt-1), cnt <= kG (uniform
// across the warp).  All loads are issued before any arithmetic.  The result
// for row round_row_of_lane(lane) is returned in the lanes where round_writer.
// Integer stores skip the row slots m with no row in any lane (m * kP >= cnt,
// a partial round): no loads and no arithmetic.  (The same branch around the
// float stores' loads costs more than it saves.)
//
// kIntQuery (integer stores): the caller knows the query is integer-valued (a row of
// an exact uint8 copy), so the FP32 fallback for other queries is not compiled in;
// its registers would otherwise set the kernel's count.
template <typename S, int DC, bool kIntQuery = false, typename IdFn>
__device__ __forceinline__ float dist_group(const Query<S, DC>& q, const void* base, const float2* scale,
                                            IdFn ids, int cnt, uint32_t D, uint32_t lane) {
    using Ly                 = Layout<S, DC>;
    constexpr int  M         = Ly::kM;
    const uint32_t chunks    = D / S::kElems;
    const uint64_t row_bytes = (uint64_t)D * 16u / (uint64_t)S::kElems;
    const uint32_t t         = lane % Ly::kT;
    const uint32_t g         = lane / Ly::kT;
    uint4          x[M][Ly::kCPL];
    float2         sc[M];  // scaled rows: (scale, scale^2 |codes|^2)
#pragma unroll
    for (int m = 0; m < M; ++m) {
        if (S::kInt && m * Ly::kP >= cnt) {
#pragma unroll
            for (int c = 0; c < Ly::kCPL; ++c) x[m][c] = make_uint4(0u, 0u, 0u, 0u);
            sc[m] = make_float2(0.f, 0.f);
            continue;
        }
        const int r     = m * Ly::kP + (int)g;
        const bool valid = r < cnt;
        uint32_t   id    = valid ? ids(r) : 0u;
        if constexpr (Ly::kNarrow) {
            // the lane's two chunks are adjacent: one 256-bit load when both lie in
            // the row and rows are 32-byte aligned (row bytes a multiple of 32)
            const uint32_t k0 = Ly::chunk(t, 0);
            if (valid && k0 + 1u < chunks && (row_bytes & 31u) == 0u) {
                load32(base, row_bytes, id, k0, x[m][0], x[m][1]);
            } else {
                x[m][0] = (valid && k0 < chunks) ? load16(base, row_bytes, id, k0) : make_uint4(0u, 0u, 0u, 0u);
                x[m][1] = (valid && k0 + 1u < chunks) ? load16(base, row_bytes, id, k0 + 1u)
                                                      : make_uint4(0u, 0u, 0u, 0u);
            }
        } else {
#pragma unroll
            for (int c = 0; c < Ly::kCPL; ++c) {
                uint32_t k = Ly::chunk(t, c);
                x[m][c]    = (valid && k < chunks) ? load16(base, row_bytes, id, k) : make_uint4(0u, 0u, 0u, 0u);
            }
        }
        if constexpr (S::kScaled) sc[m] = valid ? __ldg(scale + id) : make_float2(0.f, 0.f);
        else sc[m] = make_float2(1.f, 0.f);
    }
    if constexpr (S::kPQ) {
        // lane t of a group holds the codes of subspaces 16 t .. 16 t + 15 (none when
        // its chunk lies past the row: D = 384 in the 512-dimension class)
        float          v[M];
        const uint32_t k0 = Ly::chunk(t, 0);
#pragma unroll
        for (int m = 0; m < M; ++m) {
            uint32_t acc = 0;
            if (k0 < chunks) {
                const uint16_t* tb   = q.lut + 16u * kPqK * k0;
                const unsigned  w[4] = {x[m][0].x, x[m][0].y, x[m][0].z, x[m][0].w};
#pragma unroll
                for (int i = 0; i < 4; ++i) {
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc += tb[(4u * i + b) * kPqK + ((w[i] >> (8 * b)) & 0xffu)];
                }
            }
            v[m] = (float)acc;  // <= 16 * 65535: exact
        }
        return group_reduce<M, Ly::kT, float>(v, lane) * q.lut_scale;
    }
    if constexpr (S::kInt) {
        if (kIntQuery || q.qint) {
            int v[M];
#pragma unroll
            for (int m = 0; m < M; ++m) {
                v[m] = 0;
                if (m * Ly::kP >= cnt) continue;
                unsigned xx = 0u, qx = 0u;
#pragma unroll
                for (int c = 0; c < Ly::kCPL; ++c) {
                    const unsigned w[4] = {x[m][c].x, x[m][c].y, x[m][c].z, x[m][c].w};
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        xx = __dp4a(w[i], w[i], xx);
                        qx = __dp4a((unsigned)q.u[c][i], w[i], qx);
                    }
                }
                v[m] = (int)xx - 2 * (int)qx;
            }
            int y = group_reduce<M, Ly::kT, int>(v, lane);
            return (float)(y + q.qq);
        }
    }
    if constexpr (S::kScaled) {
        // sum (q - s c)^2 = |q|^2 - 2 s (q . c) + s^2 |c|^2: the codes are widened
        // unscaled, q . c runs on element pairs, each row's scale is applied once,
        // and s^2 |c|^2 is stored beside the scale (added by one lane per group)
        float2 qc[M];
#pragma unroll
        for (int m = 0; m < M; ++m) qc[m] = make_float2(0.f, 0.f);
#pragma unroll
        for (int m = 0; m < M; ++m) {
#pragma unroll
            for (int c = 0; c < Ly::kCPL; ++c) {
                float2 e[S::kElems / 2];
                S::codes2(x[m][c], e);
#pragma unroll
                for (int p = 0; p < S::kElems / 2; ++p) qc[m] = __ffma2_rn(q.f2[c][p], e[p], qc[m]);
            }
        }
        float v[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            v[m] = fmaf(-2.f * sc[m].x, qc[m].x + qc[m].y, q.qn);
            if (t == 0u) v[m] += sc[m].y;
        }
        // rounding can leave a tiny negative for a row equal to the query
        return fmaxf(group_reduce<M, Ly::kT, float>(v, lane), 0.f);
    } else if constexpr (!S::kInt && !S::kPQ) {
        float v[M];
        // (x - q)^2 on element pairs: x - q = fma(q, -1, x), then fma(d, d, acc)
        const float2 neg1 = make_float2(-1.f, -1.f);
        float2       acc[M];
#pragma unroll
        for (int m = 0; m < M; ++m) acc[m] = make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < Ly::kCPL; ++c) {
#pragma unroll
            for (int m = 0; m < M; ++m) {
                float2 e[S::kElems / 2];
                S::widen2(x[m][c], e);
#pragma unroll
                for (int p = 0; p < S::kElems / 2; ++p) {
                    const float2 d = __ffma2_rn(q.f2[c][p], neg1, e[p]);
                    acc[m]         = __ffma2_rn(d, d, acc[m]);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < M; ++m) v[m] = acc[m].x + acc[m].y;
        return group_reduce<M, Ly::kT, float>(v, lane);
    } else if constexpr (S::kInt && !kIntQuery) {
        // integer rows with a query that is not (rare): FP32 from the row bytes,
        // gathered again here (so the registers of the loads above are free on this
        // path and do not add to its peak), the query re-read through L1
        float v[M];
#pragma unroll
        for (int m = 0; m < M; ++m) {
            v[m]             = 0.f;
            const int  r     = m * Ly::kP + (int)g;
            const bool valid = r < cnt;
            const uint32_t id = valid ? ids(r) : 0u;
#pragma unroll
            for (int c = 0; c < Ly::kCPL; ++c) {
                const uint32_t k = Ly::chunk(t, c);
                if (!valid || k >= chunks) continue;
                const uint4    xr   = load16(base, row_bytes, id, k);
                const uint32_t w4[4] = {xr.x, xr.y, xr.z, xr.w};
#pragma unroll
                for (int v4 = 0; v4 < S::kElems / 4; ++v4) {
                    const float4   z = __ldg(reinterpret_cast<const float4*>(q.row + k * S::kElems) + v4);
                    const uint32_t w = w4[v4];
                    v[m]             = sqdiff(z.x, (float)(w & 0xffu), v[m]);
                    v[m]             = sqdiff(z.y, (float)((w >> 8) & 0xffu), v[m]);
                    v[m]             = sqdiff(z.z, (float)((w >> 16) & 0xffu), v[m]);
                    v[m]             = sqdiff(z.w, (float)(w >> 24), v[m]);
                }
            }
        }
        return group_reduce<M, Ly::kT, float>(v, lane);
    } else {
        return 0.f;  // not reached: an integer query took the dp4a path
    }
}

// Squared L2 from the query to rows ids(0) .. ids(cnt-1), cnt <= kG, stored to
// out[0 .. cnt).
template <typename S, int DC, bool kIntQuery = false, typename IdFn>
__device__ __forceinline__ void dist_round(const Query<S, DC>& q, const void* base, const float2* scale, IdFn ids,
                                           int cnt, uint32_t D, uint32_t lane, float* out) {
    const float    y  = dist_group<S, DC, kIntQuery>(q, base, scale, ids, cnt, D, lane);
    const uint32_t vi = round_row_of_lane<S, DC>(lane);
    if (round_writer<S, DC>(lane) && (int)vi < cnt) out[vi] = y;
}

// The PQ distance table of one query, built by its warp into `lut` (shared memory,
// [D / 8][256] u16): entry (m, k) = ||q_m - c_mk||^2 / scale, rounded, with one scale
// per query from a bound on every entry, (||q_m|| + max_k ||c_mk||)^2 <= 65535 scale.
// cb: [D / 8][256][8] centroids; cnorm: [D / 8] largest centroid norm per subspace.
template <int DC>
__device__ __forceinline__ void build_pq_lut(Query<StorePQ, DC>& q, uint16_t* lut, const float* cb,
                                             const float* cnorm, const float* row, uint32_t D, uint32_t lane) {
    const uint32_t M     = D / kPqSub;
    float          bound = 0.f;
    for (uint32_t m = lane; m < M; m += 32) {
        const float4 a  = __ldg(reinterpret_cast<const float4*>(row + kPqSub * m));
        const float4 b  = __ldg(reinterpret_cast<const float4*>(row + kPqSub * m) + 1);
        const float  qn = sqrtf(a.x * a.x + a.y * a.y + a.z * a.z + a.w * a.w + b.x * b.x + b.y * b.y +
                                b.z * b.z + b.w * b.w);
        const float  bm = qn + __ldg(cnorm + m);
        bound           = fmaxf(bound, bm * bm);
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) bound = fmaxf(bound, __shfl_xor_sync(0xffffffffu, bound, o));
    const float scale = bound > 0.f ? bound / 65535.f : 1.f;
    const float inv   = 1.f / scale;
    for (uint32_t e = lane; e < M * kPqK; e += 32) {
        const uint32_t m  = e / kPqK;
        const float4   qa = __ldg(reinterpret_cast<const float4*>(row + kPqSub * m));
        const float4   qb = __ldg(reinterpret_cast<const float4*>(row + kPqSub * m) + 1);
        const float4   ca = __ldg(reinterpret_cast<const float4*>(cb + (uint64_t)kPqSub * e));
        const float4   cc = __ldg(reinterpret_cast<const float4*>(cb + (uint64_t)kPqSub * e) + 1);
        float          d  = 0.f;
        d                 = sqdiff(qa.x, ca.x, d);
        d                 = sqdiff(qa.y, ca.y, d);
        d                 = sqdiff(qa.z, ca.z, d);
        d                 = sqdiff(qa.w, ca.w, d);
        d                 = sqdiff(qb.x, cc.x, d);
        d                 = sqdiff(qb.y, cc.y, d);
        d                 = sqdiff(qb.z, cc.z, d);
        d                 = sqdiff(qb.w, cc.w, d);
        lut[e]            = (uint16_t)fminf(65535.f, rintf(d * inv));
    }
    __syncwarp();
    q.lut       = lut;
    q.lut_scale = scale;
}

// Exponent e with |x| < 2^e for every x of a column whose largest magnitude has
// these float bits (0 for an all-zero column): the column's fixed-point grid is
// 2^(e - B) (exact integer sums of the medoid's column means and of PQ centroids).
__device__ __forceinline__ int column_exponent(uint32_t bound_bits) {
    if (bound_bits == 0u) return 0;
    int e = 0;
    frexpf(__uint_as_float(bound_bits), &e);  // bound < 2^e
    return e;
}

// ---------------------------------------------------------------- launches
// Blocks per SM of a launch, and the shared-memory carveout set to the smallest
// one that still holds them.  The rest of the SM's unified L1/shared memory
// stays L1, where register spills and the rows and lists that several warps
// touch are cached.
template <typename K>
inline cudaError_t fit_carveout(K kern, int threads, size_t smem, int* per_sm) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, threads, smem);
    if (e != cudaSuccess || *per_sm < 1) return e;
    int dev = 0, cap = 0, rsv = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&cap, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess) return e;
    const size_t need = (size_t)*per_sm * (smem + (size_t)rsv);
    const int    pct  = (int)((need * 100 + (size_t)cap - 1) / (size_t)cap);
    if (pct >= 100) return cudaSuccess;
    if ((e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct)) != cudaSuccess) return e;
    int check = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&check, kern, threads, smem)) != cudaSuccess) return e;
    if (check < *per_sm)  // a coarser carveout step than asked for: keep all of it
        return cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared);
    return cudaSuccess;
}

// kern<<<grid, block, smem, st>>>(args...).  With pdl, the launch is a programmatic
// dependent of the kernel before it on the stream: its blocks may be scheduled once
// every block of that kernel has executed griddepcontrol.launch_dependents (or
// exited), so their launch overlaps its end; a dependent reads that kernel's output
// only after griddepcontrol.wait, which returns when it has completed and its
// writes are visible.  Without pdl, griddepcontrol.wait returns at once.
template <typename... P, typename... A>
inline cudaError_t launch_kernel(void (*kern)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, bool pdl,
                                 A&&... args) {
    if (!pdl) {
        kern<<<grid, block, smem, st>>>(std::forward<A>(args)...);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim          = grid;
    cfg.blockDim         = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream           = st;
    cudaLaunchAttribute at[1];
    at[0].id                                         = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs                                        = at;
    cfg.numAttrs                                     = 1;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_may_launch() { asm volatile("griddepcontrol.launch_dependents;"); }

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

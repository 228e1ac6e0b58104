// staged.cu -- searchPoints2's merge of graph results with the insert list.
//
// Restates merge_and_rerank_kernel (vamana/include/utils.cuh:199-285) with the
// same decisions.  For each query the L graph worklist entries, then every staged
// (insert-list) row, compete for L slots in that order.  A candidate enters when its
// squared distance is strictly below the largest slot value, replacing the first
// slot that holds it.  The slots start at +inf and are finally put in stable
// distance order (the reference's bubble sort).
//
// The reference runs this on one thread per query.  Here one warp serves a query:
//   * each lane computes one candidate's distance, sequentially over the dimensions
//     with one fused multiply-add each, as l2_distance_sq (:150-158) compiles;
//   * a ballot of the 32 candidates against the current largest slot value selects
//     the few that can enter; they are applied in arrival order;
//   * after each replacement the (largest value, first slot) pair is rebuilt by a
//     warp reduction from per-lane maxima, where only the owning lane rescans.
#include "common.cuh"
#include "kernels.h"

namespace vann {
namespace {

constexpr uint32_t kStaged = 0x80000000u;

__device__ __forceinline__ float l2_seq(const float* q, const float* row, uint32_t D) {
    float d = 0.f;
    for (uint32_t i = 0; i < D; i += 4) {
        const float4 x = __ldg(reinterpret_cast<const float4*>(row + i));
        float        e = q[i] - x.x;
        d              = fmaf(e, e, d);
        e              = q[i + 1] - x.y;
        d              = fmaf(e, e, d);
        e              = q[i + 2] - x.z;
        d              = fmaf(e, e, d);
        e              = q[i + 3] - x.w;
        d              = fmaf(e, e, d);
    }
    return d;
}

// (largest value, first slot holding it) over the warp; v = lane's largest, s = its slot
__device__ __forceinline__ void warp_argmax(float& v, uint32_t& s) {
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const float    ov = __shfl_xor_sync(0xffffffffu, v, o);
        const uint32_t os = __shfl_xor_sync(0xffffffffu, s, o);
        if (ov > v || (ov == v && os < s)) {
            v = ov;
            s = os;
        }
    }
}

__global__ void __launch_bounds__(128) staged_merge_kernel(StagedArgs a, uint32_t warp_bytes) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib  = threadIdx.x >> 5;
    const uint32_t L = a.L, D = a.D;
    unsigned char* base = smem + (size_t)wib * warp_bytes;
    float*         qv   = reinterpret_cast<float*>(base);            // D
    float*         sd   = qv + D;                                    // p2 slot values (keys reuse)
    uint32_t*      sid  = reinterpret_cast<uint32_t*>(sd + a.p2);    // p2
    uint64_t*      keys = reinterpret_cast<uint64_t*>(sid + a.p2);   // p2
    const uint64_t total = (uint64_t)L + a.n_stage;

    for (uint64_t qi = blockIdx.x * (uint64_t)(blockDim.x / 32) + wib; qi < a.nq;
         qi += (uint64_t)gridDim.x * (blockDim.x / 32)) {
        for (uint32_t i = lane; i < D; i += 32) qv[i] = a.queries[qi * D + i];
        for (uint32_t k = lane; k < L; k += 32) {
            sd[k]  = __int_as_float(0x7f800000);  // +inf
            sid[k] = kNone;
        }
        __syncwarp();
        // this lane's slots are lane, lane + 32, ...: their largest value, first slot
        float    lmax = lane < L ? __int_as_float(0x7f800000) : -1.f;
        uint32_t lslot = lane < L ? lane : kNone;
        float    gmax  = lmax;
        uint32_t gslot = lslot;
        warp_argmax(gmax, gslot);

        for (uint64_t c0 = 0; c0 < total; c0 += 32) {
            const uint64_t c  = c0 + lane;
            float          d  = __int_as_float(0x7f800000);
            uint32_t       id = kNone;
            if (c < L) {
                id = a.graph_ids[qi * L + c];
                if (id != kNone) d = l2_seq(qv, a.vecs + (uint64_t)id * D, D);
            } else if (c < total) {
                const uint64_t s = c - L;
                id               = kStaged | (uint32_t)s;
                d                = l2_seq(qv, a.stage + s * D, D);
            }
            uint32_t m = __ballot_sync(0xffffffffu, d < gmax);
            while (m) {
                const uint32_t src = __ffs(m) - 1u;
                m &= m - 1u;
                const float dc = __shfl_sync(0xffffffffu, d, src);
                if (!(dc < gmax)) continue;  // the largest value dropped meanwhile
                const uint32_t idc = __shfl_sync(0xffffffffu, id, src);
                if (lane == (gslot & 31u)) {
                    sd[gslot]  = dc;
                    sid[gslot] = idc;
                    lmax       = -1.f;
                    lslot      = kNone;
                    for (uint32_t k = lane; k < L; k += 32)
                        if (sd[k] > lmax) {
                            lmax  = sd[k];
                            lslot = k;
                        }
                }
                gmax  = lmax;
                gslot = lslot;
                warp_argmax(gmax, gslot);
            }
        }
        __syncwarp();
        // stable order by distance: keys (distance bits, slot); +inf slots sort last
        for (uint32_t k = lane; k < a.p2; k += 32)
            keys[k] = k < L ? ((uint64_t)__float_as_uint(sd[k]) << 32) | k : ~0ull;
        __syncwarp();
        warp_bitonic_sort_smem(keys, a.p2, lane);
        for (uint32_t t = lane; t < L; t += 32) {
            const uint32_t k  = (uint32_t)keys[t];
            const uint32_t id = sid[k];
            a.out_ids[qi * L + t] = id;
            a.out_d[qi * L + t]   = sd[k];
        }
        __syncwarp();
        if (a.out_vecs) {
            for (uint32_t t = 0; t < L; ++t) {
                const uint32_t id  = sid[(uint32_t)keys[t]];
                float*         dst = a.out_vecs + (qi * L + t) * D;
                const float*   src = id == kNone ? nullptr
                                     : (id & kStaged) ? a.stage + (uint64_t)(id & ~kStaged) * D
                                                      : a.vecs + (uint64_t)id * D;
                for (uint32_t i = lane; i < D; i += 32) dst[i] = src ? __ldg(src + i) : 0.f;
            }
        }
        __syncwarp();
    }
}

}  // namespace

cudaError_t launch_staged_merge(const StagedArgs& args, int num_sms, cudaStream_t st) {
    if (args.nq == 0 || args.L == 0) return cudaSuccess;
    StagedArgs a = args;
    uint32_t   p2 = 32;
    while (p2 < a.L) p2 <<= 1;
    a.p2 = p2;
    const uint32_t warp_bytes = (4u * a.D + 4u * p2 + 4u * p2 + 8u * p2 + 15u) & ~15u;
    const int      warps      = 4;
    const size_t   smem       = (size_t)warp_bytes * warps;
    cudaError_t    e = cudaFuncSetAttribute(staged_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e          = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, staged_merge_kernel, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * num_sms;
    const uint64_t need = (a.nq + warps - 1) / warps;
    if (grid > need) grid = need;
    staged_merge_kernel<<<(unsigned)grid, warps * 32, smem, st>>>(a, warp_bytes);
    return cudaGetLastError();
}

}  // namespace vann

// prune_rev.cu -- the reverse-edge re-prune for alpha-consistent lists, one warp
// per node.
//
// After a batch, each node v that received reverse entries is re-pruned over
// A = its new reverse sources and B = its current out-neighbours
// (pruneReverseEdges, vamana/include/kernels.cuh:626-743; candidate order and the
// rule as in prune.cu).  When B came out of RobustPrune with the same alpha, no
// B candidate prunes another, so the selection only needs the distances that
// involve an A candidate: |A| x |C| of them, not |C|^2.
//
//   1. one pass of gathers gives d(v, c) for every candidate; one more per A
//      candidate gives d(a, c) (the rows are in L1 by then);
//   2. the candidates are ordered by (distance, index): B is already in that order
//      (it is a RobustPrune selection), so the A candidates are merged in by rank;
//   3. bit masks over the sorted positions: PA[i] = what A_i prunes,
//      SB[i] = the B candidates that prune A_i;
//   4. selection, all on those masks: every live B candidate ahead of the next
//      live A candidate is chosen in one step; that A candidate is chosen unless
//      a chosen B candidate prunes it, and then removes what it prunes.
// This gives the same list as evaluating every pair (prune.cu).  Distances use the
// exact uint8 rows when they are exact (dp4a), else the FP32 rows, in the same
// summation order as prune_kernel.  Nodes with more than kMaxC candidates or
// kMaxA reverse sources are handed on in out_list.
#include "common.cuh"
#include "kernels.h"

namespace vann {
namespace {

constexpr uint32_t kMaxC = 128;  // candidates per node
constexpr uint32_t kMaxA = 8;    // reverse sources per node
constexpr uint32_t kW    = kMaxC / 32;

struct RevWarp {  // shared memory of one warp
    uint32_t cid[kMaxC];
    float    cd[kMaxC];
    uint64_t keys[kMaxC];
    float    ad[kMaxA][kMaxC];  // d(A_i, candidate j)
    uint32_t pa[kMaxA][kW];     // sorted positions A_i prunes
    uint32_t sb[kMaxA][kW];     // sorted positions of B candidates that prune A_i
};

// d(row `qid`, candidate j) for every candidate j < nc into out[j]; the query comes
// from the row format the distances use (uint8 rows: the exact uint8 row itself)
template <typename S, int DC>
__device__ __forceinline__ void dists_to(const PruneArgs& a, const void* store, uint32_t qid, const uint32_t* cid,
                                         uint32_t nc, float* out, uint32_t lane) {
    Query<S, DC> q;
    if constexpr (S::kInt) load_query_u8row<S, DC>(q, a.vecs_u8 + (uint64_t)qid * a.D, a.D, lane);
    else load_query<S, DC>(q, a.vecs + (uint64_t)qid * a.D, a.D, lane);
    constexpr int G = Layout<S, DC>::kG;
    for (uint32_t g0 = 0; g0 < nc; g0 += G) {
        const int gc = (int)min((uint32_t)G, nc - g0);
        // uint8 rows are used only when every row is exact, so the query row is integer-valued
        dist_round<S, DC, S::kInt>(q, store, nullptr, [&](int j) { return cid[g0 + j]; }, gc, a.D, lane, out + g0);
    }
}

template <typename S, int DC>
__device__ __forceinline__ void all_dists(const PruneArgs& a, const void* store, RevWarp& w, uint32_t node,
                                          uint32_t nA, uint32_t nc, uint32_t lane) {
    dists_to<S, DC>(a, store, node, w.cid, nc, w.cd, lane);
    for (uint32_t i = 0; i < nA; ++i) dists_to<S, DC>(a, store, w.cid[i], w.cid, nc, w.ad[i], lane);
}

// U8: distances from the exact uint8 rows (chosen on the host, which has read the
// exactness flag); the kernel then holds one distance path only, which keeps its code
// small enough for the instruction cache.  Should the flag say otherwise on the device,
// every node is handed on to the next pass.
template <int DC, bool U8>
__global__ void __launch_bounds__(128) prune_rev_kernel(PruneArgs a, uint32_t* out_list, uint32_t* out_count) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t lane = threadIdx.x & 31u;
    RevWarp&       w    = reinterpret_cast<RevWarp*>(smem_raw)[threadIdx.x >> 5];
    const uint32_t R    = a.R;
    const bool     gated = U8 && (a.vecs_u8 == nullptr || a.gate == nullptr ||
                                  *reinterpret_cast<volatile const uint32_t*>(a.gate) != 0u);
    uint32_t       done = 0;

    for (;;) {
        uint32_t s = 0;
        if (lane == 0) s = atomicAdd(a.counter, 1u);
        s = __shfl_sync(0xffffffffu, s, 0);
        if (s >= a.n_nodes) break;
        const uint32_t node = __ldg(a.node_ids + s);
        if (node == kNone) continue;  // the padded slots' run in the sorted edge list
        const uint32_t ci   = a.csr_by_slot ? s : node;
        const uint32_t nA   = min(__ldg(a.csr_cnt + ci), a.cap);
        const uint32_t aoff = __ldg(a.csr_off + ci);
        const uint32_t nB   = a.use_b ? min(a.deg[node], R) : 0u;
        const uint32_t nc   = nA + nB;
        if (nc > kMaxC || nA > kMaxA || gated) {
            if (lane == 0) out_list[atomicAdd(out_count, 1u)] = s;
            continue;
        }
        for (uint32_t i = lane; i < nc; i += 32)
            w.cid[i] = i < nA ? __ldg(a.csr_src + aoff + i) : a.adj[(uint64_t)node * R + (i - nA)];
        __syncwarp();

        // --- 1. distances
        if constexpr (U8) all_dists<StoreU8, DC>(a, a.vecs_u8, w, node, nA, nc, lane);
        else all_dists<StoreF32, DC>(a, a.vecs, w, node, nA, nc, lane);
        __syncwarp();

        // --- 2. stable order by (distance, candidate index)
        uint32_t p2 = 32;
        while (p2 < nc) p2 <<= 1;
        // B came out of RobustPrune in selection order: nondecreasing distance, ties in
        // list order, which is also their index order here.  Then the order is B with
        // the A candidates merged in (every A index is below every B index):
        //   B_j goes to j + #{i : d(A_i) <= d(B_j)},
        //   A_i to #{j : d(B_j) < d(A_i)} + #{k : (d(A_k), k) < (d(A_i), i)}.
        // A list out of order (a graph set from outside) takes the bitonic sort.
        bool in_order = true;
        for (uint32_t j = lane; j + 1u < nB; j += 32) in_order &= w.cd[nA + j] <= w.cd[nA + j + 1u];
        if (__all_sync(0xffffffffu, in_order)) {
            for (uint32_t j = lane; j < nB; j += 32) {
                const float d   = w.cd[nA + j];
                uint32_t    pos = j;
                for (uint32_t i = 0; i < nA; ++i) pos += w.cd[i] <= d ? 1u : 0u;
                w.keys[pos] = make_key(d, nA + j);
            }
            for (uint32_t i = 0; i < nA; ++i) {
                const float di  = w.cd[i];
                uint32_t    pos = 0;
                for (uint32_t j0 = 0; j0 < nB; j0 += 32) {
                    const uint32_t j = j0 + lane;
                    pos += __popc(__ballot_sync(0xffffffffu, j < nB && w.cd[nA + j] < di));
                }
                for (uint32_t k = 0; k < nA; ++k) {
                    const float dk = w.cd[k];
                    pos += (dk < di || (dk == di && k < i)) ? 1u : 0u;
                }
                if (lane == 0) w.keys[pos] = make_key(di, i);
            }
            for (uint32_t i = nc + lane; i < p2; i += 32) w.keys[i] = ~0ull;
            __syncwarp();
        } else {
            for (uint32_t i = lane; i < p2; i += 32) w.keys[i] = i < nc ? make_key(w.cd[i], i) : ~0ull;
            __syncwarp();
            warp_bitonic_sort_smem(w.keys, p2, lane);
        }
        const uint32_t m = min(nc, a.cap);

        // --- 3. masks over sorted positions t < m (position t = 32k + lane)
        uint32_t am[kW];  // positions holding A candidates
#pragma unroll
        for (uint32_t k = 0; k < kW; ++k) {
            const uint32_t t   = 32u * k + lane;
            const uint32_t idx = t < m ? (uint32_t)w.keys[t] : 0u;
            am[k]              = __ballot_sync(0xffffffffu, t < m && idx < nA);
        }
        for (uint32_t i = 0; i < nA; ++i) {
            const float di = w.cd[i];
#pragma unroll
            for (uint32_t k = 0; k < kW; ++k) {
                const uint32_t t   = 32u * k + lane;
                bool           pr = false, by = false;
                if (t < m) {
                    const uint32_t idx = (uint32_t)w.keys[t];
                    const float    y   = w.ad[i][idx] * a.alpha;
                    pr                 = y <= w.cd[idx];           // A_i prunes the candidate at t
                    by                 = idx >= nA && y <= di;     // the B candidate at t prunes A_i
                }
                const uint32_t bp = __ballot_sync(0xffffffffu, pr), bb = __ballot_sync(0xffffffffu, by);
                if (lane == 0) {
                    w.pa[i][k] = bp;
                    w.sb[i][k] = bb;
                }
            }
        }
        __syncwarp();

        // --- 4. selection (the same on every lane)
        uint32_t live[kW], chosen_b[kW];
#pragma unroll
        for (uint32_t k = 0; k < kW; ++k) {
            const uint32_t lo = 32u * k;
            live[k]           = m >= lo + 32u ? ~0u : (m > lo ? (1u << (m - lo)) - 1u : 0u);
            chosen_b[k]       = 0u;
        }
        uint32_t       ndeg = 0;
        const uint64_t out  = (uint64_t)node * R;
        for (;;) {
            uint32_t tA = m;  // next live A candidate
#pragma unroll
            for (int k = kW - 1; k >= 0; --k)
                if (live[k] & am[k]) tA = 32u * (uint32_t)k + __ffs(live[k] & am[k]) - 1u;
            // live B candidates ahead of it: all chosen, in order, up to R
            uint32_t run[kW], total = 0;
#pragma unroll
            for (uint32_t k = 0; k < kW; ++k) {
                const uint32_t lo   = 32u * k;
                const uint32_t mask = tA >= lo + 32u ? ~0u : (tA > lo ? (1u << (tA - lo)) - 1u : 0u);
                run[k]              = live[k] & ~am[k] & mask;
                total += __popc(run[k]);
            }
            const uint32_t take = min(total, R - ndeg);
            {  // lane l writes the run members at positions 32k + l
                uint32_t rank = 0;
#pragma unroll
                for (uint32_t k = 0; k < kW; ++k) {
                    if ((run[k] >> lane) & 1u) {
                        const uint32_t r = rank + __popc(run[k] & ((1u << lane) - 1u));
                        if (r < take) {
                            const uint32_t id = w.cid[(uint32_t)w.keys[32u * k + lane]];
                            a.adj[out + ndeg + r]   = id;
                            a.adj_h[out + ndeg + r] = bloom_pack(id);
                        }
                    }
                    rank += __popc(run[k]);
                }
            }
            ndeg += take;
            if (ndeg >= R || tA >= m) break;
#pragma unroll
            for (uint32_t k = 0; k < kW; ++k) {
                chosen_b[k] |= run[k];
                live[k] &= ~run[k];
            }
            // decide the A candidate at tA
            const uint32_t i = (uint32_t)w.keys[tA];
            bool           pruned = false;
#pragma unroll
            for (uint32_t k = 0; k < kW; ++k) pruned |= (w.sb[i][k] & chosen_b[k]) != 0u;
#pragma unroll
            for (uint32_t k = 0; k < kW; ++k)
                if (k == (tA >> 5)) live[k] &= ~(1u << (tA & 31u));
            if (!pruned) {
                if (lane == 0) {
                    const uint32_t id       = w.cid[i];
                    a.adj[out + ndeg]   = id;
                    a.adj_h[out + ndeg] = bloom_pack(id);
                }
                if (++ndeg >= R) break;
#pragma unroll
                for (uint32_t k = 0; k < kW; ++k) live[k] &= ~w.pa[i][k];
            }
        }
        if (lane == 0) a.deg[node] = ndeg;
        ++done;
        __syncwarp();
    }
    if (lane == 0 && a.pruned && done) atomicAdd(a.pruned + 1, (unsigned long long)done);
}

}  // namespace

cudaError_t launch_prune_rev(const PruneArgs& a, bool u8, uint32_t* out_list, uint32_t* out_count, int num_sms,
                             cudaStream_t st) {
    if (a.n_nodes == 0) return cudaSuccess;
    if (!a.node_ids || !a.csr_off || !a.consistent || a.D > 256) return cudaErrorInvalidValue;
    const int    warps = 4;
    const size_t smem  = sizeof(RevWarp) * warps;
    auto         kern  = a.D <= 128 ? (u8 ? prune_rev_kernel<0, true> : prune_rev_kernel<0, false>)
                                    : (u8 ? prune_rev_kernel<1, true> : prune_rev_kernel<1, false>);
    cudaError_t  e     = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e          = fit_carveout(kern, warps * 32, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * num_sms;
    const uint64_t need = (a.n_nodes + warps - 1) / warps;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, warps * 32, smem, st>>>(a, out_list, out_count);
    return cudaGetLastError();
}

}  // namespace vann

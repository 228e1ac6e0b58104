// prune.cu -- RobustPrune, one warp per node, candidates staged in shared memory.
//
// Restates pruneOutNeighbors / pruneReverseEdges (vamana/include/kernels.cuh:
// 232-356, 626-743) together with the candidate preparation that the reference
// spreads over getNeighbors, computeDists, sortByDistance and the two merge
// kernels (:141-229, :567-624):
//   A = the node's expansion list (out-prune) or its reverse sources (re-prune),
//   B = the node's current out-neighbours,
//   candidates = stable sort of A then B by distance to the node (A first on
//   equal distance), truncated to `cap`;
//   repeat: p* = first INIT candidate -> out-neighbour; every INIT candidate p
//   with dist(p*, p) * alpha <= dist(node, p) becomes PRUNED; until R
//   neighbours or no INIT candidate is left.
// Distances are squared FP32.  One key (distance bits, candidate index) per
// candidate gives the stable order in a single bitonic sort.  When B is known
// to be alpha-consistent (it is the output of an earlier RobustPrune with the
// same alpha, kept in selection order), a B candidate can never be pruned by a
// B p*, so those pairs are not evaluated: the decisions are the same, the
// distance evaluations drop from |C|^2 to about |A| * |C|.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace vann {

constexpr uint8_t kInit = 0, kPruned = 1, kNeighbor = 2, kFromA = 0x10;

struct PruneLayout {
    uint32_t p2;     // sort size (power of two >= max candidates)
    uint32_t bytes;  // per warp
    static PruneLayout make(uint32_t max_cand, uint32_t R) {
        PruneLayout l;
        uint32_t    p = 32;
        while (p < max_cand) p <<= 1;
        l.p2    = p;
        l.bytes = 8u * p + 4u * p + 4u * p + p + 4u * R + 4u * 32u;
        l.bytes = (l.bytes + 15u) & ~15u;
        return l;
    }
};

template <int DC>
__global__ void __launch_bounds__(128) prune_kernel(PruneArgs a, uint32_t p2, uint32_t warp_bytes,
                                                    uint32_t chunk) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t wib  = threadIdx.x >> 5;
    unsigned char* base = smem + (size_t)wib * warp_bytes;
    uint64_t*      keys = reinterpret_cast<uint64_t*>(base);
    uint32_t*      cid  = reinterpret_cast<uint32_t*>(base + 8u * p2);
    float*         cd   = reinterpret_cast<float*>(base + 12u * p2);
    uint32_t*      sid  = reinterpret_cast<uint32_t*>(cd);  // sorted ids reuse cd
    uint8_t*       st   = base + 16u * p2;
    uint32_t*      chosen = reinterpret_cast<uint32_t*>(base + 17u * p2);
    const uint32_t R    = a.R;
    uint32_t*      plist  = chosen + R;  // positions of one round's candidates
    const bool     rev  = a.csr_off != nullptr;
    // every node, or the nodes other kernels handed over (large ones: one per warp)
    const bool     all   = a.in_count == nullptr;
    const uint64_t nwork = all ? a.n_nodes : (uint64_t)*reinterpret_cast<volatile const uint32_t*>(a.in_count);
    if (!all) chunk = 1u;

    uint32_t done = 0;  // nodes pruned by this warp
    for (;;) {
        uint32_t w0 = 0;
        if (lane == 0) w0 = atomicAdd(a.counter, chunk);
        w0 = __shfl_sync(0xffffffffu, w0, 0);
        if (w0 >= nwork) break;
        uint32_t wend = (uint32_t)min((uint64_t)w0 + chunk, nwork);
        // which of the chunk's nodes have work
        uint32_t wi   = w0 + lane;
        bool     has  = lane < chunk && wi < wend;
        uint32_t myslot = 0, mynode = 0;
        if (has) {
            myslot = all ? wi : __ldg(a.in_list + wi);
            mynode = a.node_ids ? __ldg(a.node_ids + myslot) : myslot;
            if (mynode == kNone) has = false;  // padded slots' run in the sorted edge list
            if (has && rev && a.skip_empty && __ldg(a.csr_cnt + (a.csr_by_slot ? myslot : mynode)) == 0u)
                has = false;
        }
        uint32_t todo = __ballot_sync(0xffffffffu, has);
        while (todo) {
            const uint32_t src  = __ffs(todo) - 1u;
            todo &= todo - 1u;
            const uint32_t w    = __shfl_sync(0xffffffffu, myslot, src);
            const uint32_t node = __shfl_sync(0xffffffffu, mynode, src);

            Query<StoreF32, DC> nv;
            load_query<StoreF32, DC>(nv, a.vecs + (uint64_t)node * a.D, a.D, lane);

            // --- candidates: A then B
            uint32_t nA = 0, aoff = 0;
            if (rev) {
                const uint32_t ci = a.csr_by_slot ? w : node;
                nA   = __ldg(a.csr_cnt + ci);
                aoff = __ldg(a.csr_off + ci);
                nA   = min(nA, a.cap);
            } else {
                nA = min(__ldg(a.a_n + w), a.a_stride);
            }
            uint32_t nB = a.use_b ? min(__ldg(a.deg + node), R) : 0u;
            uint32_t nc = nA + nB;
            for (uint32_t i = lane; i < nc; i += 32) {
                uint32_t id;
                float    d = 0.f;
                if (i < nA) {
                    if (rev) {
                        id = __ldg(a.csr_src + aoff + i);
                    } else {
                        id = __ldg(a.a_ids + (uint64_t)w * a.a_stride + i);
                        if (a.a_d) d = __ldg(a.a_d + (uint64_t)w * a.a_stride + i);
                    }
                } else {
                    id = __ldg(a.adj + (uint64_t)node * R + (i - nA));
                }
                cid[i] = id;
                cd[i]  = d;
            }
            __syncwarp();
            // distances to the node for the reverse sources and B
            const uint32_t dstart = (rev || a.a_d == nullptr) ? 0u : nA;
            constexpr int  G      = Layout<StoreF32, DC>::kG;
            for (uint32_t g0 = dstart; g0 < nc; g0 += G) {
                int      gc = (int)min((uint32_t)G, nc - g0);
                float    y  = dist_group<StoreF32, DC>(nv, a.vecs, nullptr,
                                                       [&](int j) { return cid[g0 + j]; }, gc, a.D, lane);
                uint32_t vi = round_row_of_lane<StoreF32, DC>(lane);
                if (round_writer<StoreF32, DC>(lane) && (int)vi < gc) cd[g0 + vi] = y;
            }
            __syncwarp();
            uint32_t ns = 32;
            while (ns < nc) ns <<= 1;
            for (uint32_t i = lane; i < ns; i += 32) keys[i] = i < nc ? make_key(cd[i], i) : ~0ull;
            __syncwarp();
            warp_bitonic_sort_smem(keys, ns, lane);
            const uint32_t ncap = min(nc, a.cap);
            for (uint32_t t = lane; t < ncap; t += 32) {
                uint32_t idx = (uint32_t)keys[t];
                sid[t]       = cid[idx];
                st[t]        = idx < nA ? kFromA : 0;
            }
            __syncwarp();

            // --- RobustPrune
            uint32_t ndeg = 0, first = 0;
            while (ndeg < R) {
                int found = -1;
                for (uint32_t c0 = first; c0 < ncap; c0 += 32) {
                    uint32_t i  = c0 + lane;
                    bool     in = i < ncap && (st[i] & 3u) == kInit;
                    uint32_t m  = __ballot_sync(0xffffffffu, in);
                    if (m) {
                        found = (int)(c0 + __ffs(m) - 1);
                        break;
                    }
                }
                if (found < 0) break;
                const uint32_t ps    = sid[found];
                const bool     ps_a  = (st[found] & kFromA) != 0;
                __syncwarp();
                if (lane == 0) {
                    st[found]    = (uint8_t)(kNeighbor | (ps_a ? kFromA : 0));
                    chosen[ndeg] = ps;
                }
                ++ndeg;
                first = (uint32_t)found + 1u;
                __syncwarp();
                if (ndeg >= R) break;

                // p*'s row is fetched only if some candidate needs its distance
                // (with consistent B lists a B p* only checks the A candidates)
                Query<StoreF32, DC> pv;
                bool                have_pv = false;
                for (uint32_t c0 = first; c0 < ncap; c0 += 32) {
                    uint32_t i    = c0 + lane;
                    bool     need = false;
                    if (i < ncap) {
                        uint8_t s = st[i];
                        need      = (s & 3u) == kInit && (!a.consistent || ps_a || (s & kFromA));
                    }
                    uint32_t m  = __ballot_sync(0xffffffffu, need);
                    uint32_t nm = __popc(m);
                    if (nm == 0) continue;
                    if (!have_pv) {
                        load_query<StoreF32, DC>(pv, a.vecs + (uint64_t)ps * a.D, a.D, lane);
                        have_pv = true;
                    }
                    if (need) plist[__popc(m & ((1u << lane) - 1u))] = i;
                    __syncwarp();
                    for (uint32_t g0 = 0; g0 < nm; g0 += G) {
                        int      gc = (int)min((uint32_t)G, nm - g0);
                        float    y  = dist_group<StoreF32, DC>(
                            pv, a.vecs, nullptr, [&](int j) { return sid[plist[g0 + j]]; }, gc, a.D, lane);
                        uint32_t vi = round_row_of_lane<StoreF32, DC>(lane);
                        if (round_writer<StoreF32, DC>(lane) && (int)vi < gc) {
                            uint32_t t = plist[g0 + vi];
                            if (y * a.alpha <= key_dist(keys[t])) st[t] = (uint8_t)(kPruned | (st[t] & kFromA));
                        }
                    }
                    __syncwarp();
                }
            }
            // rewrite the node's adjacency (in place, like the reference)
            for (uint32_t t = lane; t < ndeg; t += 32) {
                a.adj[(uint64_t)node * R + t]   = chosen[t];
                a.adj_h[(uint64_t)node * R + t] = bloom_pack(chosen[t]);
            }
            if (lane == 0) a.deg[node] = ndeg;
            __syncwarp();
            ++done;
        }
    }
    if (lane == 0 && a.pruned && done) atomicAdd(a.pruned + 1, (unsigned long long)done);
}

cudaError_t launch_prune(const PruneArgs& a, int num_sms, cudaStream_t st) {
    if (a.n_nodes == 0) return cudaSuccess;
    uint32_t    maxa = a.csr_off ? a.cap : a.a_stride;
    PruneLayout lay  = PruneLayout::make(maxa + a.R, a.R);
    const int   warps = 4;
    size_t      smem  = (size_t)lay.bytes * warps;
    void (*kern)(PruneArgs, uint32_t, uint32_t, uint32_t);
    if (a.D <= 128)
        kern = prune_kernel<0>;
    else if (a.D <= 256)
        kern = prune_kernel<1>;
    else
        kern = prune_kernel<2>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = fit_carveout(kern, warps * 32, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    // nodes per counter grab: up to 32, fewer when the launch has too few nodes to
    // give every resident warp work (each warp prunes its nodes one after another)
    const uint64_t resident = (uint64_t)per_sm * num_sms * warps;
    uint32_t       chunk    = (uint32_t)std::min<uint64_t>(32, std::max<uint64_t>(1, a.n_nodes / (4 * resident)));
    uint64_t need = (a.n_nodes + (uint64_t)chunk * warps - 1) / ((uint64_t)chunk * warps);
    uint64_t grid = (uint64_t)per_sm * num_sms;
    if (grid > need) grid = need;
    kern<<<(unsigned)grid, warps * 32, smem, st>>>(a, lay.p2, lay.bytes, chunk);
    return cudaGetLastError();
}

}  // namespace vann

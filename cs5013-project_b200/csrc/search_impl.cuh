// search.cu -- persistent batched GreedySearch, one warp per query.
//
// Restates the reference's GreedySearch (vamana/include/search.cuh:20-367):
// worklist of L entries seeded with the entry point (visited, not in the bloom
// filter), repeated expansion of the closest unvisited entry, neighbours
// filtered by the tombstones, the optional batch-index quirk and a per-query
// bloom filter (39,988 slots, two hashes), merged stably (existing entries
// before new ones on equal distance) and truncated to L.  Where the reference
// runs four kernels and a blocking host poll per hop, this kernel keeps the
// whole search of a query inside one warp: the bloom filter (bit-packed, 5 KB),
// the worklist and the hop's candidates live in shared memory, termination is
// decided on the device, and warps pull queries from a counter until none are
// left.  Every neighbour check of one expansion reads the filter as it stood
// before the expansion (the reference's filterNeighbors checks all R slots
// before any thread's mark lands; this reproduces its golden graph).
#pragma once
#include "common.cuh"
#include "kernels.h"

namespace vann {

struct SmemLayout {
    uint32_t lp;      // L rounded up to 32
    uint32_t maxr;    // neighbour slots
    uint32_t keys;    // rerank key slots (power of two) or 0
    uint32_t lut;     // offset of the PQ distance table (lut_bytes, 0 for other stores)
    uint32_t bytes;   // per warp
    __host__ __device__ static SmemLayout make(uint32_t L, uint32_t maxr, bool rerank, uint32_t lut_bytes = 0) {
        SmemLayout s;
        s.lp   = (L + 31u) & ~31u;
        s.maxr = maxr;
        s.keys = 0;
        if (rerank) {
            uint32_t p = 32;
            while (p < s.lp) p <<= 1;
            s.keys = p;
        }
        s.lut   = 5008u + 8u * s.lp + 8u * s.maxr + 8u * s.keys;
        s.bytes = s.lut + lut_bytes;
        return s;
    }
};

__device__ __forceinline__ uint32_t upper_bound_f(const float* a, uint32_t n, float x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t lower_bound_f(const float* a, uint32_t n, float x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// IQ: every query is a row of the exact uint8 copy (build and insert searches), so the
// distance code for other queries is left out (fewer registers).
template <typename S, int DC, int SPL, int MINB, bool IQ = false>
__global__ void __launch_bounds__(128, MINB) search_kernel(SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int    G     = Layout<S, DC>::kG;
    const uint32_t   lane  = threadIdx.x & 31u;
    const uint32_t   wib   = threadIdx.x >> 5;
    const SmemLayout lay   = SmemLayout::make(a.L, SPL * 32, a.rerank != 0, S::kPQ ? 64u * a.D : 0u);
    unsigned char*   base  = smem + (size_t)wib * lay.bytes;
    uint32_t*        bloom = reinterpret_cast<uint32_t*>(base);
    uint32_t*        wl_id = reinterpret_cast<uint32_t*>(base + 5008);
    float*           wl_d  = reinterpret_cast<float*>(base + 5008 + 4 * lay.lp);
    uint32_t*        nb_id = reinterpret_cast<uint32_t*>(base + 5008 + 8 * lay.lp);
    float*           nb_d  = reinterpret_cast<float*>(base + 5008 + 8 * lay.lp + 4 * lay.maxr);
    uint64_t*        nb_key = reinterpret_cast<uint64_t*>(nb_id);  // same bytes, after the ids/dists are read
    uint64_t*        keys  = reinterpret_cast<uint64_t*>(base + 5008 + 8 * lay.lp + 8 * lay.maxr);
    const uint32_t   R     = a.R;
    grid_dependency_wait();  // the order kernel's order and counter

    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(a.counter, 1u);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= a.nq) break;
        if (a.order != nullptr) q = __ldg(a.order + q);  // the query's index in the batch
        // per-query worklist size and result count (uneven batches), capped by the
        // launch's maximum, which sized the shared memory and the output rows
        const uint32_t L  = a.Lq != nullptr ? max(1u, min(__ldg(a.Lq + q), a.L)) : a.L;
        const uint32_t kq = a.kq != nullptr ? min(__ldg(a.kq + q), a.k) : a.k;

        Query<S, DC> qv;
        load_query<S, DC>(qv, a.queries + (uint64_t)q * a.D, a.D, lane, a.center);
        if constexpr (S::kPQ)
            build_pq_lut<DC>(qv, reinterpret_cast<uint16_t*>(base + lay.lut), a.pq_cb, a.pq_cnorm,
                             a.queries + (uint64_t)q * a.D, a.D, lane);
        for (uint32_t w = lane; w < kBloomWords; w += 32) bloom[w] = 0u;

        uint32_t skip = kNone;
        if (a.skip_mode == 1) skip = q;
        if (a.skip_mode == 2) skip = a.skip_base + q;

        // initializeWorklist: entry visited, distance computed, not in the filter
        const uint32_t entry = a.entry;
        float d0 = dist_group<S, DC, IQ>(qv, a.store, a.scale, [&](int) { return entry; }, 1, a.D, lane);
        d0       = __shfl_sync(0xffffffffu, d0, 0);  // row 0 lives in lane 0
        if (lane == 0) {
            wl_id[0] = entry | kVisitedBit;
            wl_d[0]  = d0;
        }
        __syncwarp();
        uint32_t n = 1, parent = entry, ppos = 0, hops = 0, nv = 0, evals = 1, adjw = 0;
        float    pd = d0;
        // the parent's degree, adjacency row and filter slots, loaded in one round
        // trip; from the second hop on they are prefetched before the merge
        uint32_t nid[SPL], hp[SPL], dg;
        auto     fetch_row = [&](uint32_t node) {
            const uint32_t* row  = a.adj + (uint64_t)node * R;
            const uint32_t* rowh = a.adj_h + (uint64_t)node * R;
#pragma unroll
            for (int s = 0; s < SPL; ++s) {
                uint32_t j = (uint32_t)s * 32u + lane;
                nid[s]     = j < R ? __ldg(row + j) : 0u;
                hp[s]      = j < R ? __ldg(rowh + j) : 0u;
            }
            dg = __ldg(a.deg + node);
        };
        fetch_row(parent);

        for (;;) {
            if (hops >= a.max_hops) {
                if (lane == 0) atomicOr(a.status, kStatusHopLimit);
                break;
            }
            ++hops;
            if (a.vis_ids != nullptr && nv < a.max_visited) {
                if (lane == 0) {
                    a.vis_ids[(uint64_t)q * a.max_visited + nv] = parent;
                    a.vis_d[(uint64_t)q * a.max_visited + nv]   = pd;
                }
                ++nv;
            }
            dg = dg < R ? dg : R;
            adjw += dg;

            // filterNeighbors: every slot checks the filter as it stood before this
            // expansion, then the new neighbours are marked
            uint32_t h1[SPL], h2[SPL];
            bool     pass[SPL];
#pragma unroll
            for (int s = 0; s < SPL; ++s) {
                uint32_t j  = (uint32_t)s * 32u + lane;
                bool     ok = j < dg;
                if (ok && a.tomb != nullptr) ok = !((__ldg(a.tomb + (nid[s] >> 5)) >> (nid[s] & 31u)) & 1u);
                if (ok && nid[s] == skip) ok = false;
                h1[s] = hp[s] >> 16;
                h2[s] = hp[s] & 0xffffu;
                if (ok) {
                    bool seen = ((bloom[h1[s] >> 5] >> (h1[s] & 31u)) & 1u) &&
                                ((bloom[h2[s] >> 5] >> (h2[s] & 31u)) & 1u);
                    ok = !seen;
                }
                pass[s] = ok;
            }
            __syncwarp();
            uint32_t cnt = 0;
#pragma unroll
            for (int s = 0; s < SPL; ++s) {
                if (pass[s]) {
                    atomicOr(&bloom[h1[s] >> 5], 1u << (h1[s] & 31u));
                    atomicOr(&bloom[h2[s] >> 5], 1u << (h2[s] & 31u));
                }
                uint32_t m = __ballot_sync(0xffffffffu, pass[s]);
                if (pass[s]) nb_id[cnt + __popc(m & ((1u << lane) - 1u))] = nid[s];
                cnt += __popc(m);
            }
            __syncwarp();
            evals += cnt;

            // distances: G rows per gather round, all loads of a round in flight
            for (uint32_t g0 = 0; g0 < cnt; g0 += G) {
                int   gc = (int)min((uint32_t)G, cnt - g0);
                dist_round<S, DC, IQ>(qv, a.store, a.scale, [&](int j) { return nb_id[g0 + j]; }, gc, a.D, lane,
                                      nb_d + g0);
            }
            __syncwarp();

            // candidates that cannot enter a full worklist are dropped before the
            // sort: with n == L a new entry with d >= wl_d[L-1] lands at >= L
            const float tail = n == L ? wl_d[L - 1] : __int_as_float(0x7f800000);
            uint64_t    key[SPL];
            bool        keep[SPL];
#pragma unroll
            for (int s = 0; s < SPL; ++s) {
                uint32_t j = (uint32_t)s * 32u + lane;
                keep[s]    = false;
                key[s]     = ~0ull;
                if (j < cnt) {
                    float dd = nb_d[j];
                    keep[s]  = n < L || dd < tail;
                    key[s]   = make_key(dd, nb_id[j]);
                }
            }
            __syncwarp();
            uint32_t kc = 0;
#pragma unroll
            for (int s = 0; s < SPL; ++s) {
                uint32_t m = __ballot_sync(0xffffffffu, keep[s]);
                if (keep[s]) nb_key[kc + __popc(m & ((1u << lane) - 1u))] = key[s];
                kc += __popc(m);
            }
            __syncwarp();

            if (kc > 0) {
                // sort the kept candidates by (distance, id) with the smallest network
                uint32_t n2 = 1;
                while (n2 < kc) n2 <<= 1;
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    uint32_t j = (uint32_t)s * 32u + lane;
                    key[s]     = j < kc ? nb_key[j] : ~0ull;
                }
                if (n2 > 1) {
                    if (n2 <= 32) {
                        uint64_t k1[1] = {key[0]};
                        warp_bitonic_sort<1>(k1, lane, n2);
                        key[0] = k1[0];
                    } else {
                        warp_bitonic_sort<SPL>(key, lane, n2);
                    }
                }
                __syncwarp();
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    uint32_t j = (uint32_t)s * 32u + lane;
                    if (j < kc) {
                        nb_id[j] = (uint32_t)key[s];
                        nb_d[j]  = key_dist(key[s]);
                    }
                }
                __syncwarp();

            }

            // next parent, decided before the merge: the first unvisited entry of the
            // merged list is either the best kept candidate or the first unvisited
            // existing entry after the current parent, whichever is closer (existing
            // first on equal distance).  Its row is fetched now so the load overlaps
            // the merge.
            uint32_t e_pos = kNone;
            for (uint32_t c0 = ppos + 1u; c0 < n; c0 += 32u) {
                uint32_t i  = c0 + lane;
                bool     uv = i < n && !(wl_id[i] & kVisitedBit);
                uint32_t m  = __ballot_sync(0xffffffffu, uv);
                if (m) {
                    e_pos = c0 + __ffs(m) - 1u;
                    break;
                }
            }
            const float    d_e      = e_pos != kNone ? wl_d[e_pos] : __int_as_float(0x7f800000);
            const bool     take_new = kc > 0 && nb_d[0] < d_e;
            const bool     has_next = take_new || e_pos != kNone;
            const uint32_t next     = take_new ? nb_id[0] : (has_next ? (wl_id[e_pos] & ~kVisitedBit) : 0u);
            const float    next_d   = take_new ? nb_d[0] : d_e;
            if (has_next) fetch_row(next);
            __syncwarp();

            uint32_t p0 = L;
            if (kc > 0) {
                // mergeIntoWorklist: new entry j lands at j + #(existing <= d_j);
                // existing entry i moves to i + #(new < d_i); keep the first L
                uint32_t pj[SPL];
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    uint32_t j = (uint32_t)s * 32u + lane;
                    pj[s]      = j < kc ? j + upper_bound_f(wl_d, n, nb_d[j]) : L;
                }
                p0 = __shfl_sync(0xffffffffu, pj[0], 0);
                if (p0 < L) {
                    if (p0 < n) {
                        uint32_t nchunks = (n - p0 + 31u) >> 5;
                        for (int c = (int)nchunks - 1; c >= 0; --c) {
                            uint32_t i  = p0 + (uint32_t)c * 32u + lane;
                            uint32_t id = 0, np = L;
                            float    dd = 0.f;
                            if (i < n) {
                                id = wl_id[i];
                                dd = wl_d[i];
                                np = i + lower_bound_f(nb_d, kc, dd);
                            }
                            __syncwarp();
                            if (np < L) {
                                wl_id[np] = id;
                                wl_d[np]  = dd;
                            }
                            __syncwarp();
                        }
                    }
#pragma unroll
                    for (int s = 0; s < SPL; ++s) {
                        uint32_t j = (uint32_t)s * 32u + lane;
                        if (j < kc && pj[s] < L) {
                            wl_id[pj[s]] = nb_id[j];
                            wl_d[pj[s]]  = nb_d[j];
                        }
                    }
                    n = min(n + kc, L);
                }
                __syncwarp();
            }

            if (!has_next) break;
            ppos   = take_new ? p0 : e_pos;
            parent = next;
            pd     = next_d;
            if (lane == 0) wl_id[ppos] = parent | kVisitedBit;
            __syncwarp();
        }

        // outputs
        if (a.out_ids != nullptr) {
            if (a.rerank) {
                // exact FP32 distances of the final worklist, sorted (dist, position)
                constexpr int        GF = Layout<StoreF32, DC>::kG;
                Query<StoreF32, DC> qf;
                load_query<StoreF32, DC>(qf, a.queries + (uint64_t)q * a.D, a.D, lane);
                for (uint32_t g0 = 0; g0 < n; g0 += GF) {
                    int   gc = (int)min((uint32_t)GF, n - g0);
                    float y  = dist_group<StoreF32, DC>(
                        qf, a.vecs_f32, nullptr, [&](int j) { return wl_id[g0 + j] & ~kVisitedBit; }, gc, a.D,
                        lane);
                    uint32_t vi = round_row_of_lane<StoreF32, DC>(lane);
                    if (round_writer<StoreF32, DC>(lane) && (int)vi < gc) keys[g0 + vi] = make_key(y, g0 + vi);
                }
                __syncwarp();
                for (uint32_t i = n + lane; i < lay.keys; i += 32) keys[i] = ~0ull;
                __syncwarp();
                warp_bitonic_sort_smem(keys, lay.keys, lane);
                for (uint32_t t = lane; t < a.k; t += 32) {
                    uint64_t o = (uint64_t)q * a.k + t;
                    if (t < n && t < kq) {
                        a.out_ids[o] = wl_id[(uint32_t)keys[t]] & ~kVisitedBit;
                        a.out_d[o]   = key_dist(keys[t]);
                    } else {
                        a.out_ids[o] = kNone;
                        a.out_d[o]   = __int_as_float(0x7f800000);
                    }
                }
            } else {
                for (uint32_t t = lane; t < a.k; t += 32) {
                    uint64_t o = (uint64_t)q * a.k + t;
                    if (t < n && t < kq) {
                        a.out_ids[o] = wl_id[t] & ~kVisitedBit;
                        a.out_d[o]   = wl_d[t];
                    } else {
                        a.out_ids[o] = kNone;
                        a.out_d[o]   = __int_as_float(0x7f800000);
                    }
                }
            }
        }
        if (lane == 0) {
            if (a.vis_n != nullptr) a.vis_n[q] = nv;
            if (a.hops_out != nullptr) a.hops_out[q] = hops;
            if (a.evals_out != nullptr) a.evals_out[q] = evals;
            if (a.adjw_out != nullptr) a.adjw_out[q] = adjw;
        }
        __syncwarp();
    }
}

template <typename S, int DC, int SPL, int MINB, bool IQ = false>
static cudaError_t launch_t(const SearchArgs& a, int num_sms, cudaStream_t st) {
    SmemLayout lay   = SmemLayout::make(a.L, SPL * 32, a.rerank != 0, S::kPQ ? 64u * a.D : 0u);
    const int  warps = 4;
    size_t     smem  = (size_t)lay.bytes * warps;
    auto       kern  = search_kernel<S, DC, SPL, MINB, IQ>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = fit_carveout(kern, warps * 32, smem, &per_sm);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t need = (a.nq + warps - 1) / warps;
    uint64_t grid = (uint64_t)per_sm * num_sms;
    if (grid > need) grid = need;
    if (grid == 0) return cudaSuccess;
    return launch_kernel(kern, dim3((unsigned)grid), dim3(warps * 32), smem, st, a.pdl != 0, a);
}

}  // namespace vann

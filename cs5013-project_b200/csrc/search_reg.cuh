// search_reg.cuh -- GreedySearch with the worklist held in registers (L <= 64).
//
// Same semantics as search_kernel (search_impl.cuh), restating the reference's
// GreedySearch (vamana/include/search.cuh:20-367); only the worklist differs.
// Element e of the worklist lives in lane e % 32, register e / 32, as a 64-bit
// key (distance bits << 32 | insertion sequence) and a payload (id | visited).
// Insertion sequences grow with every merge and, within one expansion, follow
// the (distance, id) order of the new candidates, so the key order is exactly
// the reference's stable merge order: equal distances keep older entries first
// (mergeIntoWorklist, search.cuh:140-223).  A merge is a half-cleaner between
// the worklist and the reversed sorted candidates followed by a bitonic merge
// network; the next parent is one ballot.
//
// BEAM = 2 is a batched form beside the reference's algorithm (not a parity
// form): each hop expands the first two unvisited entries together, so a query
// takes about half the hops, each with two lists in flight and fuller gather
// rounds.  The second list is filtered after the first one's marks, and the kept
// candidates are sorted and merged in batches of up to 64.
#pragma once
#include "search_impl.cuh"

namespace vann {

constexpr uint64_t kSentinel = ~0ull;

struct RegLayout {
    uint32_t maxr;   // candidate slots (>= 64 so that the rerank ids fit too)
    uint32_t lut;    // offset of the PQ distance table (lut_bytes of them, 0 for other stores)
    uint32_t bytes;  // per warp: bloom filter + candidate ids/distances + 64 merge payloads + table
    __host__ __device__ static RegLayout make(uint32_t slots, uint32_t lut_bytes = 0) {
        RegLayout l;
        l.maxr  = slots < 64u ? 64u : slots;
        l.lut   = 5008u + 8u * l.maxr + 256u;
        l.bytes = l.lut + lut_bytes;
        return l;
    }
};

// Kept candidates up to this count are merged by rank (below); more go through
// the bitonic sort and merge network.
constexpr uint32_t kRankMergeMax = 24;

// Merge of kc <= 32 kept candidates (keys (distance bits << 32 | id) in cand[0 .. kc),
// unsorted) into the register worklist by counting ranks: candidate j goes to
// (worklist entries at or below its distance) + (candidates before it in (distance,
// id) order); worklist entry e moves down by the candidates strictly closer.  That is
// the order the sort + merge network gives (equal distances: older entries first,
// new ones by id), in about a dozen instructions per candidate instead of two
// networks of shuffles.  Positions at or beyond L fall off; the new entries take
// insertion sequences seq + rank.  skey / spay: 64 staging slots in shared memory
// (skey may alias cand: it is written after every lane has read cand).
template <int LREG>
__device__ __forceinline__ void rank_merge(uint64_t (&wk)[LREG], uint32_t (&wp)[LREG], const uint64_t* cand,
                                           uint32_t kc, uint32_t seq, uint32_t& n, uint32_t L, uint64_t* skey,
                                           uint32_t* spay, uint32_t lane) {
    const uint64_t cj    = lane < kc ? cand[lane] : kSentinel;
    uint32_t       crank = 0, cpos = 0;
    uint32_t       wsh[LREG];
    uint32_t       wd[LREG];
#pragma unroll
    for (int r = 0; r < LREG; ++r) {
        wsh[r] = 0u;
        wd[r]  = (uint32_t)(wk[r] >> 32);  // sentinels: 0xFFFFFFFF, above every distance
    }
    for (uint32_t k = 0; k < kc; ++k) {
        const uint64_t ck = cand[k];
        const uint32_t cd = (uint32_t)(ck >> 32);
        crank += (ck < cj || (ck == cj && k < lane)) ? 1u : 0u;
        uint32_t before = 0;
#pragma unroll
        for (int r = 0; r < LREG; ++r) {
            wsh[r] += cd < wd[r] ? 1u : 0u;
            before += __popc(__ballot_sync(0xffffffffu, wd[r] <= cd));
        }
        if (lane == k) cpos = before;
    }
    __syncwarp();  // every lane has read cand: skey may overwrite it
#pragma unroll
    for (int r = 0; r < LREG; ++r) {
        const uint32_t p = (uint32_t)r * 32u + lane + wsh[r];
        if (wk[r] != kSentinel && p < L) {
            skey[p] = wk[r];
            spay[p] = wp[r];
        }
    }
    if (lane < kc) {
        const uint32_t p = cpos + crank;
        if (p < L) {
            skey[p] = (cj & 0xffffffff00000000ull) | (uint64_t)(seq + crank);
            spay[p] = (uint32_t)cj;
        }
    }
    __syncwarp();
    n = min(n + kc, L);
#pragma unroll
    for (int r = 0; r < LREG; ++r) {
        const uint32_t e = (uint32_t)r * 32u + lane;
        wk[r]            = e < n ? skey[e] : kSentinel;
        wp[r]            = e < n ? spay[e] : 0u;
    }
    __syncwarp();
}

// Lower half of the union of two ascending sequences of N = 32 * LREG keys,
// sorted ascending in place in (wk, wp).  Keys are unique except sentinels.
template <int LREG>
__device__ __forceinline__ void reg_merge(uint64_t (&wk)[LREG], uint32_t (&wp)[LREG],
                                          const uint64_t (&ck)[LREG], const uint32_t (&cp)[LREG],
                                          uint32_t lane) {
#pragma unroll
    for (int r = 0; r < LREG; ++r) {
        uint64_t rk = __shfl_sync(0xffffffffu, ck[LREG - 1 - r], 31 - lane);
        uint32_t rp = __shfl_sync(0xffffffffu, cp[LREG - 1 - r], 31 - lane);
        if (rk < wk[r]) {
            wk[r] = rk;
            wp[r] = rp;
        }
    }
    if constexpr (LREG == 2) {
        if (wk[1] < wk[0]) {
            uint64_t tk = wk[0];
            uint32_t tp = wp[0];
            wk[0] = wk[1];
            wp[0] = wp[1];
            wk[1] = tk;
            wp[1] = tp;
        }
    }
#pragma unroll
    for (int j = 16; j >= 1; j >>= 1) {
        const bool lower = (lane & (uint32_t)j) == 0;
#pragma unroll
        for (int r = 0; r < LREG; ++r) {
            uint64_t ok = __shfl_xor_sync(0xffffffffu, wk[r], j);
            uint32_t op = __shfl_xor_sync(0xffffffffu, wp[r], j);
            bool     take = lower ? (ok < wk[r]) : (ok > wk[r]);
            if (take) {
                wk[r] = ok;
                wp[r] = op;
            }
        }
    }
}

template <typename S, int DC, int SPL, int LREG, int MINB, int BEAM>
__global__ void __launch_bounds__(128, MINB) search_kernel_rw(SearchArgs a) {
    static_assert(BEAM == 1 || BEAM == 2, "one or two parents per hop");
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int   G     = Layout<S, DC>::kG;
    constexpr int   NS    = BEAM * SPL;  // neighbour slots per lane in one hop
    const uint32_t  lane  = threadIdx.x & 31u;
    const uint32_t  wib   = threadIdx.x >> 5;
    const RegLayout lay   = RegLayout::make(NS * 32, S::kPQ ? 64u * a.D : 0u);
    unsigned char*  base  = smem + (size_t)wib * lay.bytes;
    uint32_t*       bloom = reinterpret_cast<uint32_t*>(base);
    uint32_t*       nb_id = reinterpret_cast<uint32_t*>(base + 5008);
    float*          nb_d  = reinterpret_cast<float*>(base + 5008 + 4 * lay.maxr);
    uint64_t*       nb_key = reinterpret_cast<uint64_t*>(nb_id);  // after ids/dists are read
    uint32_t*       m_pay = reinterpret_cast<uint32_t*>(base + 5008 + 8 * lay.maxr);  // rank-merge payloads
    uint64_t*       rkeys = reinterpret_cast<uint64_t*>(base);     // rerank keys, after the search
    const uint32_t  R     = a.R;
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

        // initializeWorklist: the entry, visited, distance computed, not in the filter
        const uint32_t entry = a.entry;
        float d0 = dist_group<S, DC>(qv, a.store, a.scale, [&](int) { return entry; }, 1, a.D, lane);
        d0       = __shfl_sync(0xffffffffu, d0, 0);
        uint64_t wk[LREG];
        uint32_t wp[LREG];
#pragma unroll
        for (int r = 0; r < LREG; ++r) {
            wk[r] = kSentinel;
            wp[r] = 0u;
        }
        if (lane == 0) {
            wk[0] = make_key(d0, 0u);
            wp[0] = entry | kVisitedBit;
        }
        uint32_t n = 1, seq = 1, hops = 0, nv = 0, evals = 1, adjw = 0, np = 1;
        uint32_t par[BEAM];
        float    pd[BEAM];
        par[0] = entry;
        pd[0]  = d0;
        // the parents' degrees, adjacency rows and filter slots, all in one round trip
        uint32_t nid[BEAM][SPL], hp[BEAM][SPL], dg[BEAM];
        auto     fetch_rows = [&]() {
#pragma unroll
            for (int b = 0; b < BEAM; ++b) {
                const bool      live = (uint32_t)b < np;
                const uint32_t  node = live ? par[b] : 0u;
                const uint32_t* row  = a.adj + (uint64_t)node * R;
                const uint32_t* rowh = a.adj_h + (uint64_t)node * R;
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    uint32_t j = (uint32_t)s * 32u + lane;
                    nid[b][s]  = live && j < R ? __ldg(row + j) : 0u;
                    hp[b][s]   = live && j < R ? __ldg(rowh + j) : 0u;
                }
                dg[b] = live ? __ldg(a.deg + node) : 0u;
            }
        };
        fetch_rows();

        for (;;) {
            if (hops >= a.max_hops) {
                if (lane == 0) atomicOr(a.status, kStatusHopLimit);
                break;
            }
            ++hops;
            uint32_t cnt = 0;
#pragma unroll
            for (int b = 0; b < BEAM; ++b) {
                if ((uint32_t)b >= np) break;
                if (a.vis_ids != nullptr && nv < a.max_visited) {
                    if (lane == 0) {
                        a.vis_ids[(uint64_t)q * a.max_visited + nv] = par[b];
                        a.vis_d[(uint64_t)q * a.max_visited + nv]   = pd[b];
                    }
                    ++nv;
                }
                const uint32_t dgb = dg[b] < R ? dg[b] : R;
                adjw += dgb;

                // filterNeighbors: snapshot check of every slot of the list, then mark
                bool pass[SPL];
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    const uint32_t j  = (uint32_t)s * 32u + lane;
                    const uint32_t id = nid[b][s];
                    bool           ok = j < dgb;
                    if (ok && a.tomb != nullptr) ok = !((__ldg(a.tomb + (id >> 5)) >> (id & 31u)) & 1u);
                    if (ok && id == skip) ok = false;
                    if (ok) {
                        uint32_t h1 = hp[b][s] >> 16, h2 = hp[b][s] & 0xffffu;
                        ok = !(((bloom[h1 >> 5] >> (h1 & 31u)) & 1u) && ((bloom[h2 >> 5] >> (h2 & 31u)) & 1u));
                    }
                    pass[s] = ok;
                }
                __syncwarp();
#pragma unroll
                for (int s = 0; s < SPL; ++s) {
                    if (pass[s]) {
                        uint32_t h1 = hp[b][s] >> 16, h2 = hp[b][s] & 0xffffu;
                        atomicOr(&bloom[h1 >> 5], 1u << (h1 & 31u));
                        atomicOr(&bloom[h2 >> 5], 1u << (h2 & 31u));
                    }
                    uint32_t m = __ballot_sync(0xffffffffu, pass[s]);
                    if (pass[s]) nb_id[cnt + __popc(m & ((1u << lane) - 1u))] = nid[b][s];
                    cnt += __popc(m);
                }
                __syncwarp();
            }
            evals += cnt;

            for (uint32_t g0 = 0; g0 < cnt; g0 += G) {
                int      gc = (int)min((uint32_t)G, cnt - g0);
                dist_round<S, DC>(qv, a.store, a.scale, [&](int j) { return nb_id[g0 + j]; }, gc, a.D, lane,
                                  nb_d + g0);
            }
            __syncwarp();

            // keep the candidates that can enter the list, compacted to nb_key
            float tail = __int_as_float(0x7f800000);
            if (n == L) {
                const int last = (int)L - 1;
                uint64_t  mine = wk[0];
#pragma unroll
                for (int r = 1; r < LREG; ++r)
                    if (r == last / 32) mine = wk[r];
                tail = key_dist(__shfl_sync(0xffffffffu, mine, last % 32));
            }
            uint64_t ckey[NS];
            bool     keep[NS];
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                uint32_t j = (uint32_t)s * 32u + lane;
                keep[s]    = false;
                ckey[s]    = kSentinel;
                if (j < cnt) {
                    float dd = nb_d[j];
                    keep[s]  = dd < tail;
                    ckey[s]  = make_key(dd, nb_id[j]);
                }
            }
            __syncwarp();
            uint32_t kc = 0;
#pragma unroll
            for (int s = 0; s < NS; ++s) {
                uint32_t m = __ballot_sync(0xffffffffu, keep[s]);
                if (keep[s]) nb_key[kc + __popc(m & ((1u << lane) - 1u))] = ckey[s];
                kc += __popc(m);
            }
            __syncwarp();

            if (BEAM == 1 && kc > 0u && kc <= kRankMergeMax) {
                rank_merge<LREG>(wk, wp, nb_key, kc, seq, n, L, nb_key, m_pay, lane);
                seq += kc;
                kc = 0u;  // merged
            }
            // at most 64 kept candidates per batch (one batch unless BEAM = 2)
            for (uint32_t b0 = 0; b0 < kc; b0 += 64u) {
                const uint32_t  bc = min(64u, kc - b0);
                const uint64_t* bk = nb_key + b0;
                // sort the kept candidates by (distance, id); only the best N can enter
                uint64_t ck[LREG];
                uint32_t cp[LREG];
                if (bc <= 32) {
                    uint64_t k1[1] = {lane < bc ? bk[lane] : kSentinel};
                    uint32_t n2    = 1;
                    while (n2 < bc) n2 <<= 1;
                    if (n2 > 1) warp_bitonic_sort<1>(k1, lane, n2);
                    ck[0] = k1[0];
                    if constexpr (LREG == 2) ck[1] = kSentinel;
                } else {
                    uint64_t k2[2];
                    k2[0] = bk[lane];
                    k2[1] = lane + 32u < bc ? bk[lane + 32u] : kSentinel;
                    warp_bitonic_sort<2>(k2, lane, 64u);
                    ck[0] = k2[0];
                    if constexpr (LREG == 2) ck[1] = k2[1];
                }
                // worklist keys: distance bits, then the next insertion sequence
#pragma unroll
                for (int r = 0; r < LREG; ++r) {
                    uint32_t e = (uint32_t)r * 32u + lane;
                    if (ck[r] != kSentinel && e < bc) {
                        cp[r] = (uint32_t)ck[r];
                        ck[r] = (ck[r] & 0xffffffff00000000ull) | (uint64_t)(seq + e);
                    } else {
                        cp[r] = 0u;
                        ck[r] = kSentinel;
                    }
                }
                seq += bc;
                reg_merge<LREG>(wk, wp, ck, cp, lane);
                n = min(n + bc, L);
#pragma unroll
                for (int r = 0; r < LREG; ++r) {
                    if ((uint32_t)r * 32u + lane >= L) {  // truncate to L
                        wk[r] = kSentinel;
                        wp[r] = 0u;
                    }
                }
            }
            __syncwarp();

            // next parents: the first BEAM unvisited entries, in list order
            int      fr[BEAM], fl[BEAM];
            uint32_t got = 0;
#pragma unroll
            for (int b = 0; b < BEAM; ++b) {
                fr[b] = -1;
                fl[b] = 0;
            }
#pragma unroll
            for (int r = 0; r < LREG; ++r) {
                uint32_t m = __ballot_sync(0xffffffffu, wk[r] != kSentinel && !(wp[r] & kVisitedBit));
#pragma unroll
                for (int b = 0; b < BEAM; ++b) {
                    if (m != 0u && got < (uint32_t)BEAM) {
                        const int l = __ffs(m) - 1;
                        m &= m - 1u;
                        if (got == 0u) {
                            fr[0] = r;
                            fl[0] = l;
                        } else {
                            fr[BEAM - 1] = r;
                            fl[BEAM - 1] = l;
                        }
                        ++got;
                    }
                }
            }
            if (got == 0u) break;
            np = got;
#pragma unroll
            for (int b = 0; b < BEAM; ++b) {
                if (fr[b] < 0) continue;
                uint32_t pk_lo = 0;
                uint64_t pkey  = 0;
#pragma unroll
                for (int r = 0; r < LREG; ++r) {
                    uint32_t p  = __shfl_sync(0xffffffffu, wp[r], fl[b]);
                    uint64_t kk = __shfl_sync(0xffffffffu, wk[r], fl[b]);
                    if (r == fr[b]) {
                        pk_lo = p;
                        pkey  = kk;
                    }
                }
#pragma unroll
                for (int r = 0; r < LREG; ++r)
                    if (r == fr[b] && lane == (uint32_t)fl[b]) wp[r] |= kVisitedBit;
                par[b] = pk_lo & ~kVisitedBit;
                pd[b]  = key_dist(pkey);
            }
            fetch_rows();
        }

        // outputs
        if (a.out_ids != nullptr) {
            if (a.rerank) {
                // exact FP32 distances of the final worklist, sorted (dist, position)
#pragma unroll
                for (int r = 0; r < LREG; ++r) {
                    uint32_t e = (uint32_t)r * 32u + lane;
                    if (e < n) nb_id[e] = wp[r] & ~kVisitedBit;
                }
                __syncwarp();
                constexpr int       GF = Layout<StoreF32, DC>::kG;
                Query<StoreF32, DC> qf;
                load_query<StoreF32, DC>(qf, a.queries + (uint64_t)q * a.D, a.D, lane);
                for (uint32_t g0 = 0; g0 < n; g0 += GF) {
                    int   gc = (int)min((uint32_t)GF, n - g0);
                    float y  = dist_group<StoreF32, DC>(qf, a.vecs_f32, nullptr,
                                                        [&](int j) { return nb_id[g0 + j]; }, gc, a.D, lane);
                    uint32_t vi = round_row_of_lane<StoreF32, DC>(lane);
                    if (round_writer<StoreF32, DC>(lane) && (int)vi < gc) rkeys[g0 + vi] = make_key(y, g0 + vi);
                }
                __syncwarp();
                uint32_t ns = 32;
                while (ns < n) ns <<= 1;
                for (uint32_t i = n + lane; i < ns; i += 32) rkeys[i] = kSentinel;
                __syncwarp();
                warp_bitonic_sort_smem(rkeys, ns, lane);
                for (uint32_t t = lane; t < a.k; t += 32) {
                    uint64_t o = (uint64_t)q * a.k + t;
                    if (t < n && t < kq) {
                        a.out_ids[o] = nb_id[(uint32_t)rkeys[t]];
                        a.out_d[o]   = key_dist(rkeys[t]);
                    } else {
                        a.out_ids[o] = kNone;
                        a.out_d[o]   = __int_as_float(0x7f800000);
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < LREG; ++r) {
                    uint32_t e = (uint32_t)r * 32u + lane;
                    if (e < a.k) {
                        uint64_t o   = (uint64_t)q * a.k + e;
                        a.out_ids[o] = e < n && e < kq ? (wp[r] & ~kVisitedBit) : kNone;
                        a.out_d[o]   = e < n && e < kq ? key_dist(wk[r]) : __int_as_float(0x7f800000);
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

template <typename S, int DC, int SPL, int LREG, int MINB, int BEAM = 1>
static cudaError_t launch_rw(const SearchArgs& a, int num_sms, cudaStream_t st) {
    RegLayout  lay   = RegLayout::make(BEAM * SPL * 32, S::kPQ ? 64u * a.D : 0u);
    const int  warps = 4;
    size_t     smem  = (size_t)lay.bytes * warps;
    auto       kern  = search_kernel_rw<S, DC, SPL, LREG, MINB, BEAM>;
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

// prune_tc.cu -- RobustPrune with the candidates' Gram matrix on the tensor cores.
//
// Same decisions as prune_kernel (prune.cu), which restates pruneOutNeighbors /
// pruneReverseEdges (vamana/include/kernels.cuh:232-356, 626-743), for indexes
// whose rows are integers in [0, 255] held exactly in the uint8 copy.  For such
// rows every squared distance is an integer below 2^24 when D <= 256, so FP32
// sums in any order, and the integer identity |x|^2 + |y|^2 - 2 x.y, give the
// same value: the decisions are bit-identical to the FP32 path.
//
// One CTA of 4 warps prunes one node at a time:
//   1. candidate ids (A then B, as in prune.cu) with their distances to the node
//      (given by the search, or computed exactly from the uint8 rows);
//   2. stable order by (distance, candidate index): each key's rank is the count
//      of smaller keys (one pass, one barrier);
//   3. the first `cap` candidates' uint8 rows are staged in shared memory in that
//      order, in the K-major no-swizzle layout tcgen05.mma reads (8-row x 16-byte
//      core matrices), and one thread issues tcgen05.mma.kind::i8 (u8 x u8 -> s32)
//      for the Gram matrix G = C C^T into tensor memory (TMEM), 128 x <= 128 per tile;
//   4. thread t reads TMEM lane t (row t of G) and writes the bit mask of the
//      candidates u that t, once chosen, prunes: alpha * d(t, u) <= d(node, u);
//   5. one warp runs the sequential selection on bits only: p* = first live
//      candidate, then the live set loses p*'s mask.  No row is fetched there.
// Nodes with more than 256 candidates go to a second pass of the same kernel with
// room for 512, larger ones to prune_kernel.  If the uint8 copy is not exact (a device flag written by
// the conversion kernels) this kernel returns at once and prune_kernel does all.
#include "common.cuh"
#include "kernels.h"

namespace vann {
namespace {

constexpr uint32_t kThreads  = 128;  // 4 warps = the 128 TMEM lanes
constexpr uint32_t kTmemCols = 128;  // accumulator columns per CTA
constexpr uint32_t kMaxR     = 128;
constexpr long long kSpinCycles = 2000000000ll;  // ~1 s bound on an MMA completion wait

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo = byte distance
// between the two 16-byte K chunks of one MMA, sbo = between 8-row groups
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: D s32, A and B unsigned 8-bit, both K-major
__device__ __forceinline__ uint32_t idesc_u8(uint32_t M, uint32_t N) {
    return (2u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_u8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive columns of this thread's TMEM lane; the wait is in the same asm
// statement so no use of r can be scheduled before the data has arrived
__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15])
        : "r"(addr)
        : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the MMA commit of the given phase
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try(bar, parity))
        if (clock64() - t0 > kSpinCycles) return false;
    return true;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint32_t dp4a_u(uint32_t a, uint32_t b, uint32_t c) { return __dp4a(a, b, c); }

// shared memory of one CTA handling up to maxc candidates per node
struct TcLayout {
    uint32_t rows, nodev, cid, cd, keys, perm, sid, sd, nrm, pm, bmask, bar, misc, bytes;
    __host__ __device__ static TcLayout make(uint32_t D, uint32_t maxc) {
        TcLayout l;
        l.rows  = 0;                  // maxc x D bytes, canonical layout, sorted order
        l.nodev = l.rows + maxc * D;  // D bytes
        l.cid   = l.nodev + ((D + 15) & ~15u);
        l.cd    = l.cid + 4 * maxc;   // candidate order (A then B)
        l.keys  = l.cd + 4 * maxc;    // 8-byte aligned: every offset above is a multiple of 16
        l.perm  = l.keys + 8 * maxc;  // sorted position -> candidate index
        l.sid   = l.perm + 4 * maxc;  // ids, distances, squared norms in sorted order
        l.sd    = l.sid + 4 * maxc;
        l.nrm   = l.sd + 4 * maxc;
        l.pm    = l.nrm + 4 * maxc;   // [maxc][maxc / 32] prune masks
        l.bmask = l.pm + maxc * maxc / 8;  // sorted positions holding B candidates
        l.bar   = l.bmask + maxc / 8;
        l.misc  = l.bar + 8;
        l.bytes = l.misc + 4 * 16;
        return l;
    }
};

__device__ __forceinline__ uint64_t u64_of(uint32_t lo, uint32_t hi) { return ((uint64_t)hi << 32) | lo; }

// Nodes are the slots in_list[0 .. *in_count) (or 0 .. n_nodes when in_list is
// null); nodes with more than MAXC candidates go to out_list.
template <uint32_t MAXC>
__global__ void __launch_bounds__(kThreads) prune_tc_kernel(PruneArgs a, uint32_t* counter, const uint32_t* in_list,
                                                            const uint32_t* in_count, uint32_t* out_list,
                                                            uint32_t* out_count) {
    constexpr uint32_t QW  = MAXC / 32;        // mask words per candidate
    constexpr uint32_t NB  = MAXC / 128;       // 128-row blocks
    constexpr uint32_t KPT = MAXC / kThreads;  // sort keys per thread
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const uint64_t nwork = in_list ? (uint64_t)*reinterpret_cast<volatile const uint32_t*>(in_count) : a.n_nodes;
    if (nwork == 0) return;
    if (*reinterpret_cast<volatile const uint32_t*>(a.gate) != 0u) {  // rows not exact: hand every node on
        for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + tid; i < nwork; i += (uint64_t)gridDim.x * blockDim.x)
            out_list[atomicAdd(out_count, 1u)] = in_list ? __ldg(in_list + i) : (uint32_t)i;
        return;
    }

    const uint32_t D = a.D, R = a.R;
    const TcLayout lay = TcLayout::make(D, MAXC);
    unsigned char* rows  = smem + lay.rows;
    uint8_t*       nodev = smem + lay.nodev;
    uint32_t*      cid   = reinterpret_cast<uint32_t*>(smem + lay.cid);
    float*         cd    = reinterpret_cast<float*>(smem + lay.cd);
    uint64_t*      keys  = reinterpret_cast<uint64_t*>(smem + lay.keys);
    uint32_t*      perm  = reinterpret_cast<uint32_t*>(smem + lay.perm);
    uint32_t*      sid   = reinterpret_cast<uint32_t*>(smem + lay.sid);
    float*         sd    = reinterpret_cast<float*>(smem + lay.sd);
    uint32_t*      nrm   = reinterpret_cast<uint32_t*>(smem + lay.nrm);
    uint32_t*      pm    = reinterpret_cast<uint32_t*>(smem + lay.pm);
    uint32_t*      bmask = reinterpret_cast<uint32_t*>(smem + lay.bmask);
    uint32_t*      misc  = reinterpret_cast<uint32_t*>(smem + lay.misc);  // [0] tmem, [2..13] work items
    const uint32_t bar    = saddr(smem + lay.bar);
    const uint32_t rows_s = saddr(rows);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(misc)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = misc[0];

    const bool     rev    = a.csr_off != nullptr;
    const uint32_t nchunk = D / 16;
    const uint32_t LBO = 128, SBO = 8 * D;  // 8 rows x 16 B per core matrix; chunks adjacent
    const uint32_t ksteps = D / 32;         // kind::i8: K = 32 per instruction
    uint32_t       phase  = 0;
    bool           failed = false;
    uint32_t       done   = 0;  // nodes pruned by this CTA

    // The next work item (slot, node, |A|, A offset, |B|) is fetched by one thread
    // while the CTA prunes the current one, so its chain of dependent loads (work
    // counter, node id, list bounds, degree) is off the critical path.
    auto fetch = [&](uint32_t* item) {
        uint32_t       w = kNone, node = kNone, nA = 0, aoff = 0, nB = 0;
        const uint32_t i = atomicAdd(counter, 1u);
        if (i < nwork) {
            w    = in_list ? __ldg(in_list + i) : i;
            node = a.node_ids ? __ldg(a.node_ids + w) : w;  // kNone: the padded slots' run
            if (node != kNone) {
                if (rev) {
                    const uint32_t ci = a.csr_by_slot ? w : node;
                    nA                = __ldg(a.csr_cnt + ci);
                    aoff              = __ldg(a.csr_off + ci);
                    if (a.skip_empty && nA == 0u) node = kNone;
                    nA = min(nA, a.cap);
                } else {
                    nA = min(__ldg(a.a_n + w), a.a_stride);
                }
                if (node != kNone && a.use_b) nB = min(a.deg[node], R);
            }
        }
        item[0] = w;
        item[1] = node;
        item[2] = nA;
        item[3] = aoff;
        item[4] = nB;
    };
    if (tid == 32) fetch(misc + 2);
    __syncthreads();

    for (uint32_t it = 0;; ++it, __syncthreads()) {
        const uint32_t* cur  = misc + 2 + 6 * (it & 1u);
        const uint32_t  w    = cur[0];
        const uint32_t  node = cur[1];
        const uint32_t  nA = cur[2], aoff = cur[3], nB = cur[4];
        if (w == kNone) break;
        if (tid == 32) fetch(misc + 2 + 6 * ((it + 1u) & 1u));
        if (node == kNone) continue;
        const uint32_t nc = nA + nB;
        if (nc > MAXC) {
            if (tid == 0) out_list[atomicAdd(out_count, 1u)] = w;
            continue;
        }
        const bool computed = rev || nB > 0 || a.a_d == nullptr;  // some distance is not given

        // --- 1. candidate ids (A then B) and given distances; the node's row
        for (uint32_t i = tid; i < nc; i += kThreads) {
            uint32_t id;
            float    d = -1.f;  // computed below
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
        if (computed && tid < nchunk)
            *reinterpret_cast<uint4*>(nodev + 16 * tid) =
                __ldg(reinterpret_cast<const uint4*>(a.vecs_u8 + (uint64_t)node * D) + tid);
        __syncthreads();

        // --- 2. missing distances straight from the uint8 rows (exact integers)
        if (computed) {
            uint32_t nn = 0;  // |node|^2
            for (uint32_t c = 0; c < nchunk; ++c) {
                const uint4 q = *reinterpret_cast<const uint4*>(nodev + 16 * c);
                nn = dp4a_u(q.x, q.x, dp4a_u(q.y, q.y, dp4a_u(q.z, q.z, dp4a_u(q.w, q.w, nn))));
            }
            for (uint32_t i = tid; i < nc; i += kThreads) {
                if (cd[i] >= 0.f) continue;
                const uint4* row = reinterpret_cast<const uint4*>(a.vecs_u8 + (uint64_t)cid[i] * D);
                uint32_t     n = 0, dot = 0;
                for (uint32_t c = 0; c < nchunk; ++c) {
                    const uint4 v = __ldg(row + c);
                    const uint4 q = *reinterpret_cast<const uint4*>(nodev + 16 * c);
                    n   = dp4a_u(v.x, v.x, dp4a_u(v.y, v.y, dp4a_u(v.z, v.z, dp4a_u(v.w, v.w, n))));
                    dot = dp4a_u(v.x, q.x, dp4a_u(v.y, q.y, dp4a_u(v.z, q.z, dp4a_u(v.w, q.w, dot))));
                }
                cd[i] = (float)(nn + n - 2u * dot);
            }
        }
        for (uint32_t i = tid; i < nc; i += kThreads) keys[i] = make_key(cd[i], i);
        if (tid == 0 && (nc & 1u)) keys[nc] = ~0ull;  // pairs below read one past an odd count
        __syncthreads();

        // --- 3. stable order by (distance, candidate index): rank = keys below
        {
            uint64_t k[KPT];
            uint32_t r[KPT];
#pragma unroll
            for (uint32_t q = 0; q < KPT; ++q) {
                const uint32_t i = tid + q * kThreads;
                k[q]             = i < nc ? keys[i] : ~0ull;
                r[q]             = 0;
            }
            const uint32_t used = (nc + kThreads - 1) / kThreads;  // key slots in use per thread
            for (uint32_t j = 0; j < nc; j += 2) {
                const uint4    kk = *reinterpret_cast<const uint4*>(keys + j);
                const uint64_t x = u64_of(kk.x, kk.y), y = u64_of(kk.z, kk.w);
#pragma unroll
                for (uint32_t q = 0; q < KPT; ++q)
                    if (q < used) r[q] += (uint32_t)(x < k[q]) + (uint32_t)(y < k[q]);
            }
#pragma unroll
            for (uint32_t q = 0; q < KPT; ++q) {
                const uint32_t i = tid + q * kThreads;
                if (i < nc) perm[r[q]] = i;
            }
        }
        __syncthreads();

        // --- 4. the first ncap candidates in sorted order: rows staged for the MMA
        const uint32_t m = min(nc, a.cap);
#pragma unroll
        for (uint32_t q = 0; q < NB; ++q) {
            const uint32_t t = 128u * q + tid;
            bool           b = false;
            if (t < m) {
                const uint32_t i = perm[t];
                sid[t]           = cid[i];
                sd[t]            = cd[i];
                b                = i >= nA;
            }
            const uint32_t bits = __ballot_sync(0xffffffffu, b);
            if (lane == 0) bmask[4u * q + warp] = bits;
        }
        for (uint32_t x = tid; x < m * nchunk; x += kThreads) {
            const uint32_t t = x / nchunk, c = x - t * nchunk;
            cp_async16(rows_s + (t >> 3) * SBO + c * LBO + (t & 7u) * 16u,
                       a.vecs_u8 + (uint64_t)cid[perm[t]] * D + 16u * c);
        }
        cp_async_wait_all();
        fence_proxy_async();  // rows become visible to the tensor core's reads
        __syncthreads();

        // --- 5. Gram tiles on the tensor cores; squared norms of the staged rows
        const uint32_t nb = (m + 127u) / 128u;  // row / column blocks of 128
        auto issue_tile = [&](uint32_t r, uint32_t c) {
            const uint32_t left = m - 128u * c;
            const uint32_t N    = ((left < 128u ? left : 128u) + 15u) & ~15u;
            const uint32_t id   = idesc_u8(128u, N);
            for (uint32_t s = 0; s < ksteps; ++s) {
                const uint64_t da = umma_desc(rows_s + r * 16u * SBO + s * 2u * LBO, LBO, SBO);
                const uint64_t db = umma_desc(rows_s + c * 16u * SBO + s * 2u * LBO, LBO, SBO);
                mma_u8(tmem, da, db, id, s > 0 ? 1u : 0u);
            }
            mma_commit(bar);
        };
        if (m > 0 && tid == 0) {
            tc_fence_after();
            issue_tile(0, 0);
        }
        for (uint32_t t = tid; t < m; t += kThreads) {
            uint32_t n = 0;
            for (uint32_t c = 0; c < nchunk; ++c) {
                const uint4 v = *reinterpret_cast<const uint4*>(rows + (t >> 3) * SBO + c * LBO + (t & 7u) * 16u);
                n = dp4a_u(v.x, v.x, dp4a_u(v.y, v.y, dp4a_u(v.z, v.z, dp4a_u(v.w, v.w, n))));
            }
            nrm[t] = n;
            // "t prunes u" is alpha * d(t, u) <= d(node, u) in FP32, with d(t, u) the exact
            // integer Y = |t|^2 + |u|^2 - 2 t.u (< 2^24, so FP32 holds it exactly).  fl(Y *
            // alpha) does not decrease as Y grows, so the test is Y <= Ymax(u), the largest
            // integer with fl(Ymax * alpha) <= d(node, u): 2 t.u - |t|^2 >= |u|^2 - Ymax(u).
            // That threshold replaces d(node, u) in the same slot.
            const float sdt = sd[t];
            int         y   = (int)fminf(floorf(sdt / a.alpha), 16777215.f);
            while (y < 16777215 && (float)(y + 1) * a.alpha <= sdt) ++y;
            while (y > 0 && (float)y * a.alpha > sdt) --y;
            reinterpret_cast<int*>(sd)[t] = (int)n - y;
        }
        __syncthreads();
        const int* thr = reinterpret_cast<const int*>(sd);

        // --- 6. prune masks in sorted order: bit u of row t = "t, once chosen, prunes u"
        for (uint32_t r = 0; r < nb; ++r) {
            const uint32_t t  = 128u * r + tid;
            const int      nt = t < m ? (int)nrm[t] : 0;
            uint32_t       mk[QW];
#pragma unroll
            for (uint32_t q = 0; q < QW; ++q) mk[q] = 0u;
#pragma unroll
            for (uint32_t c = 0; c < NB; ++c) {
                if (c < nb) {
                    if (r != 0 || c != 0) {
                        tc_fence_before();
                        __syncthreads();  // every thread's reads of the previous tile are done
                        if (tid == 0) {
                            tc_fence_after();
                            issue_tile(r, c);
                        }
                    }
                    const bool ok = mbar_wait(bar, phase);
                    phase ^= 1u;
                    if (__syncthreads_or(!ok)) {
                        failed = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t left = m - 128u * c;
                    const uint32_t N    = ((left < 128u ? left : 128u) + 15u) & ~15u;
#pragma unroll
                    for (uint32_t c16 = 0; c16 < 128u; c16 += 16u) {
                        if (c16 < N) {
                            uint32_t g[16];
                            tmem_ld16(tmem + ((32u * warp) << 16) + c16, g);
                            uint32_t bits = 0;
#pragma unroll
                            for (uint32_t k = 0; k < 16; ++k) {
                                const uint32_t u = 128u * c + c16 + k;
                                bits |= (uint32_t)((int)(2u * g[k]) - nt >= thr[u]) << k;
                            }
                            mk[4u * c + (c16 >> 5)] |= bits << (c16 & 16u);
                        }
                    }
                }
            }
            if (failed) break;
            if (t < m) {
                uint4* dst = reinterpret_cast<uint4*>(pm + t * QW);
#pragma unroll
                for (uint32_t q = 0; q < QW / 4; ++q)
                    dst[q] = make_uint4(mk[4 * q], mk[4 * q + 1], mk[4 * q + 2], mk[4 * q + 3]);
            }
        }
        if (failed) break;
        tc_fence_before();
        __syncthreads();

        // --- 7. sequential selection on bits (warp 0): lane q holds live-set word q
        if (warp == 0) {
            uint32_t live = 0u;
            if (lane < QW && m > 32u * lane) {
                const uint32_t left = m - 32u * lane;
                live                = left >= 32u ? ~0u : (1u << left) - 1u;
            }
            uint64_t       out  = (uint64_t)node * R;
            uint32_t       ndeg = 0;
            auto emit = [&](uint32_t t, uint32_t slot) {
                const uint32_t id = sid[t];
                a.adj[out + slot]   = id;
                a.adj_h[out + slot] = bloom_pack(id);
            };
            if (!a.consistent) {
                // one round per chosen neighbour
                while (ndeg < R) {
                    const uint32_t bm = __ballot_sync(0xffffffffu, live != 0u);
                    if (bm == 0u) break;
                    const uint32_t k0 = __ffs(bm) - 1u;
                    const uint32_t wv = __shfl_sync(0xffffffffu, live, k0);
                    const uint32_t t  = 32u * k0 + __ffs(wv) - 1u;
                    if (lane == 0) emit(t, ndeg);
                    ++ndeg;
                    if (ndeg >= R) break;
                    if (lane < QW) live &= ~pm[t * QW + lane];
                    if (lane == k0) live &= ~(1u << (t & 31u));
                }
            } else {
                // B came out of RobustPrune with this alpha, so no B candidate prunes
                // another: every live B candidate before the next live A candidate is
                // chosen in one step, then that A candidate is decided.
                const uint32_t bw = lane < QW ? bmask[lane] : 0u;
                while (ndeg < R) {
                    const uint32_t aw  = live & ~bw;
                    const uint32_t bmA = __ballot_sync(0xffffffffu, aw != 0u);
                    uint32_t       tA  = m;
                    if (bmA) {
                        const uint32_t k = __ffs(bmA) - 1u;
                        tA               = 32u * k + __ffs(__shfl_sync(0xffffffffu, aw, k)) - 1u;
                    }
                    uint32_t run = 0u;
                    if (lane < QW) {
                        const uint32_t lo     = 32u * lane;
                        const uint32_t before = tA >= lo + 32u ? ~0u : (tA <= lo ? 0u : (1u << (tA - lo)) - 1u);
                        run                   = live & bw & before;
                    }
                    const uint32_t cnt = __popc(run);
                    uint32_t       inc = cnt;  // inclusive prefix over lanes
#pragma unroll
                    for (uint32_t o = 1; o < 32; o <<= 1) {
                        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
                        if (lane >= o) inc += v;
                    }
                    const uint32_t total = __shfl_sync(0xffffffffu, inc, 31);
                    const uint32_t take  = min(total, R - ndeg);
                    uint32_t       j     = inc - cnt;
                    for (uint32_t bits = run; bits != 0u && j < take; bits &= bits - 1u, ++j)
                        emit(32u * lane + __ffs(bits) - 1u, ndeg + j);
                    ndeg += take;
                    if (ndeg >= R) break;
                    live &= ~run;
                    uint32_t acc = 0u;  // everything the run prunes
                    for (uint32_t q = 0; q < QW; ++q) {
                        for (uint32_t rq = __shfl_sync(0xffffffffu, run, q); rq != 0u; rq &= rq - 1u) {
                            const uint32_t t = 32u * q + __ffs(rq) - 1u;
                            if (lane < QW) acc |= pm[t * QW + lane];
                        }
                    }
                    live &= ~acc;
                    if (tA >= m) break;  // every live candidate was in the run
                    const uint32_t tw = __shfl_sync(0xffffffffu, live, tA >> 5);
                    if ((tw >> (tA & 31u)) & 1u) {
                        if (lane == 0) emit(tA, ndeg);
                        ++ndeg;
                        if (ndeg >= R) break;
                        if (lane < QW) live &= ~pm[tA * QW + lane];
                        if (lane == (tA >> 5)) live &= ~(1u << (tA & 31u));
                    }
                }
            }
            if (lane == 0) a.deg[node] = ndeg;
        }
        ++done;
    }
    if (failed && tid == 0) atomicOr(a.status, kStatusTimeout);
    if (tid == 0 && a.pruned && done) atomicAdd(a.pruned, (unsigned long long)done);
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

}  // namespace

bool prune_tc_supported(uint32_t D, uint32_t R) { return D % 32 == 0 && D >= 32 && D <= 256 && R <= kMaxR; }

namespace {

template <uint32_t MAXC>
cudaError_t launch_tc(const PruneArgs& a, uint32_t* counter, const uint32_t* in_list, const uint32_t* in_count,
                      uint32_t* out_list, uint32_t* out_count, uint64_t max_nodes, int num_sms, cudaStream_t st) {
    int dev = 0, per_sm_smem = 0, reserved = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&per_sm_smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (e != cudaSuccess) return e;
    // TMEM holds 512 columns per SM: at most 512 / kTmemCols CTAs of these kernels may
    // share an SM, which the shared-memory request enforces (an extra CTA would wait
    // in tcgen05.alloc for one of the others to exit).
    const int    max_ctas    = 512 / (int)kTmemCols;
    size_t       smem        = TcLayout::make(a.D, MAXC).bytes;
    const size_t floor_bytes = (size_t)(per_sm_smem / (max_ctas + 1) - reserved + 1024);
    if (smem < floor_bytes) smem = floor_bytes;
    auto kern = prune_tc_kernel<MAXC>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    // CTAs per SM from the shared-memory budget (the occupancy query reports one CTA
    // per SM for kernels that allocate tensor memory, which is not the limit here)
    int per_sm = per_sm_smem / (int)(smem + reserved);
    if (per_sm > max_ctas) per_sm = max_ctas;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    uint64_t grid = (uint64_t)per_sm * num_sms;
    if (grid > max_nodes) grid = max_nodes;
    kern<<<(unsigned)grid, kThreads, smem, st>>>(a, counter, in_list, in_count, out_list, out_count);
    return cudaGetLastError();
}

}  // namespace

// Passes of 256 candidates (4 CTAs per SM), then 512 (2 per SM), then 768 (one per
// SM, when its shared memory fits: D <= 160), each over the nodes the previous one
// handed on.  The first pass takes in_list[0 .. *in_count) (every node when null);
// what the last cannot take goes to out_list for prune_kernel.
// ws: 2 * n_nodes + 4 words of device scratch; counters: three zeroed work counters.
cudaError_t launch_prune_tc(const PruneArgs& a, const uint32_t* in_list, const uint32_t* in_count,
                            uint32_t* out_list, uint32_t* out_count, uint32_t* ws, uint32_t* counters, int num_sms,
                            cudaStream_t st) {
    if (a.n_nodes == 0) return cudaSuccess;
    if (!prune_tc_supported(a.D, a.R) || !a.vecs_u8 || !a.gate || !out_list || !out_count)
        return cudaErrorInvalidValue;
    int dev = 0, max_optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const bool third  = TcLayout::make(a.D, 768).bytes <= (uint32_t)max_optin;
    uint32_t*  list1  = ws;
    uint32_t*  count1 = ws + a.n_nodes;
    uint32_t*  list2  = third ? ws + a.n_nodes + 1 : out_list;
    uint32_t*  count2 = third ? ws + 2 * a.n_nodes + 1 : out_count;
    for (uint32_t* c : {count1, count2, out_count}) {
        e = cudaMemsetAsync(c, 0, sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
    }
    e = launch_tc<256>(a, counters, in_list, in_count, list1, count1, a.n_nodes, num_sms, st);
    if (e != cudaSuccess) return e;
    e = launch_tc<512>(a, counters + 1, list1, count1, list2, count2, a.n_nodes, num_sms, st);
    if (e != cudaSuccess || !third) return e;
    return launch_tc<768>(a, counters + 2, list2, count2, out_list, out_count, a.n_nodes, num_sms, st);
}

}  // namespace vann

// Tensor-core form of the QuickSampling mismatch map (sm_100a, tcgen05).
//
// The cross-correlation part of a node's map, S_b(p) = sum_j sum_l
// c_{b,j,l} * layer_l(p + o_j), is, for a batch of nodes over a shared
// template prefix o_0..o_{T-1}, the product of a node matrix A (nodes x K,
// K = T x L coefficients, zero where a node has no neighbour) with the
// pattern matrix P (TI positions x K, the layers gathered at every prefix
// offset: an im2col of the training image).  One launch computes
// D = A * P^T for a node tile of 128 rows against a range of position tiles
// and keeps, per node, the W best scores of its range in a heap (the
// shortlist); nothing of D leaves the SM.
//
//   warp 0      TMA producer: A and P tiles (128-byte swizzled K blocks) into
//               a ring of shared-memory stages, completion on mbarriers
//   warp 1      TMEM allocation and the MMA issuer: tcgen05.mma (kind::f16
//               for BF16, kind::f8f6f4 for FP8 E4M3) of M=128 nodes x N=256
//               positions x K=16/32, FP32 accumulators in TMEM, two buffers
//               of 256 columns so that the epilogue of tile t overlaps the
//               MMAs of tile t+1; tcgen05.commit frees stages and buffers
//   warps 2-5   epilogue: one thread per node (TMEM lane), 32 columns per
//               tcgen05.ld; score = acc * node_scale * pos_scale + node_bias;
//               scores at least the heap's minimum go through the full key
//               (ordered score, 32-bit tie hash of node seed and position),
//               the node's validity box (the template inside the TI) and a
//               replace-root/sift-down in shared memory
//
// Every mbarrier wait is bounded by a clock budget; on expiry the kernel
// records DEV_TC_WAIT, drains the copies it issued (bounded too), frees its
// TMEM and returns.  No cluster, no multicast: every TMA load reads this
// GPU's own memory into the issuing CTA.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "qsk_internal.h"
#include "qsk_pdl.cuh"

namespace qsk {
namespace tc {

constexpr int BM = 128;                  // nodes per CTA tile (TMEM lanes)
constexpr int BN = 256;                  // positions per tile (accumulator columns)
constexpr int BKB = 128;                 // bytes of K per block: one 128-byte swizzle row
constexpr int A_BYTES = BM * BKB;        // 16 KB
constexpr int B_BYTES = BN * BKB;        // 32 KB
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
// epilogue groups: each group is four warps, one per TMEM lane quarter, and
// takes every G-th 32-column chunk of a tile with its own top-W; more groups
// hide more of the insertion latency (the W = 32 registers allow two)
__host__ __device__ constexpr int epi_groups(int W) { return W <= 16 ? 4 : 2; }
__host__ __device__ constexpr int threads_for(int W) { return 64 + 128 * epi_groups(W); }
constexpr long long WAIT_CYCLES = 4000000000LL;   // about two seconds at 1.9 GHz

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// wait for the phase of `parity` to complete, at most WAIT_CYCLES; false on expiry
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, volatile int *abort_flag) {
    if (mbar_try(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (abort_flag && *abort_flag) return false;
        if (clock64() - t0 > WAIT_CYCLES) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major operand tile in the 128-byte swizzle layout written by TMA:
// rows of 128 bytes, 8-row groups 1024 bytes apart (stride byte offset),
// leading byte offset unused for this layout, descriptor version 1 (sm_100)
__device__ __forceinline__ uint64_t sw128_desc(unsigned saddr) {
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// instruction descriptor: FP32 accumulator, A and B of format `fmt`
// (kind::f16: 1 = BF16; kind::f8f6f4: 0 = E4M3), both K-major, M x N
__host__ __device__ constexpr unsigned make_idesc(unsigned fmt, int M, int N) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (unsigned(N >> 3) << 17) | (unsigned(M >> 4) << 24);
}

template <int KIND>
__device__ __forceinline__ void mma(unsigned tmem_d, uint64_t adesc, uint64_t bdesc, unsigned idesc, unsigned acc) {
    if constexpr (KIND == 0) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
            : "memory");
    }
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 lanes x 32 consecutive 32-bit columns of TMEM into registers
__device__ __forceinline__ void tmem_ld32(unsigned taddr, float (&v)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// monotone map of a float to an unsigned (NaN and -inf lowest)
__device__ __forceinline__ unsigned ordered(float f) {
    if (f != f) return 0u;
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(unsigned o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

// insert key (larger than k[0]) into the ascending register array k of W
// keys, dropping the minimum: the new key replaces k[0] and bubbles up by
// compare-and-swap steps (no branch, no memory)
template <int W>
__device__ __forceinline__ void sorted_insert(unsigned long long (&k)[W], unsigned (&p)[W], unsigned long long key,
                                              unsigned pos) {
    k[0] = key;
    p[0] = pos;
#pragma unroll
    for (int i = 0; i + 1 < W; ++i) {
        const bool sw = k[i] > k[i + 1];
        const unsigned long long a = k[i], b = k[i + 1];
        const unsigned pa = p[i], pb = p[i + 1];
        k[i] = sw ? b : a;
        k[i + 1] = sw ? a : b;
        p[i] = sw ? pb : pa;
        p[i + 1] = sw ? pa : pb;
    }
}

template <int KIND, int W, int STAGES>
__global__ void __launch_bounds__(threads_for(W), 1)
    k_tc_shortlist(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_p, TcArgs a) {
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte aligned stage ring (the swizzle atom), then heaps and barriers
    const unsigned raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *sA = smem;                                   // STAGES x A_BYTES
    uint8_t *sB = smem + STAGES * A_BYTES;                // STAGES x B_BYTES
    constexpr int G = epi_groups(W), EPI_WARPS = 4 * G, THREADS = threads_for(W);
    // the other epilogue groups' W best per node, for the final merge: [group-1][entry][row]
    unsigned long long *hk = reinterpret_cast<unsigned long long *>(smem + STAGES * STAGE_BYTES);
    unsigned *hp = reinterpret_cast<unsigned *>(hk + (G - 1) * W * BM);
    uint64_t *bar = reinterpret_cast<uint64_t *>(hp + (G - 1) * W * BM);
    uint64_t *full = bar, *empty = bar + STAGES, *tfull = bar + 2 * STAGES, *tempty = tfull + 2, *done = tempty + 2;
    __shared__ unsigned tmem_base_s;
    __shared__ volatile int abort_s;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile_m = blockIdx.x, range = blockIdx.y;
    const long long t_begin = (long long)range * a.tiles_per_range;
    long long t_end = t_begin + a.tiles_per_range;
    if (t_end > a.n_tiles) t_end = a.n_tiles;
    const int nkb = a.tile_kblocks ? a.tile_kblocks[tile_m] : a.kblocks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], EPI_WARPS);
        }
        mbar_init(done, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tmem_base_s))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_base_s;
    // launched programmatically after the kernel that writes A and the
    // per-node bounds: the set-up above overlaps its end, nothing below
    // reads or writes global memory before it has completed
    griddep_wait();
    griddep_launch();

    if (warp == 0) {
        // ---------------- TMA producer ----------------
        if (lane == 0 && t_begin < t_end && nkb > 0) {
            int s = 0;
            unsigned ph = 0;
            unsigned issued_ph[STAGES];
            bool pending[STAGES];
            for (int i = 0; i < STAGES; ++i) pending[i] = false;
            bool ok = true;
            for (long long t = t_begin; t < t_end && ok; ++t) {
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(&empty[s], ph ^ 1u, &abort_s)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    tma_load_2d(sA + s * A_BYTES, &map_a, &full[s], kb * a.k_per_block, tile_m * BM);
                    tma_load_2d(sB + s * B_BYTES, &map_p, &full[s], kb * a.k_per_block, (int)(t * BN));
                    pending[s] = true;
                    issued_ph[s] = ph;
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
            }
            if (!ok) {
                atomicExch(a.status, DEV_TC_WAIT);
                abort_s = 1;
            }
            // every copy issued has landed before the CTA may leave
            for (int i = 0; i < STAGES; ++i)
                if (pending[i]) mbar_wait(&full[i], issued_ph[i], nullptr);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0 && t_begin < t_end && nkb > 0) {
            constexpr unsigned idesc = make_idesc(KIND == 0 ? 1u : 0u, BM, BN);
            constexpr int KSTEPS = 4;   // 128-byte K block / 32 bytes per MMA
            int s = 0;
            unsigned ph = 0;
            bool ok = true;
            int i = 0;
            for (long long t = t_begin; t < t_end && ok; ++t, ++i) {
                const int b = i & 1;
                const unsigned tph = (unsigned)(i >> 1) & 1u;
                if (!mbar_wait(&tempty[b], tph ^ 1u, &abort_s)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const unsigned dcol = tmem + (unsigned)(b * BN);
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(&full[s], ph, &abort_s)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ad = sw128_desc(smem_u32(sA + s * A_BYTES));
                    const uint64_t bd = sw128_desc(smem_u32(sB + s * B_BYTES));
#pragma unroll
                    for (int k = 0; k < KSTEPS; ++k)
                        mma<KIND>(dcol, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), idesc, (kb | k) != 0);
                    mma_commit(&empty[s]);
                    if (++s == STAGES) {
                        s = 0;
                        ph ^= 1u;
                    }
                }
                if (ok) mma_commit(&tfull[b]);
            }
            if (!ok) {
                atomicExch(a.status, DEV_TC_WAIT);
                abort_s = 1;
            }
            // every MMA issued has completed before the TMEM is freed
            mma_commit(done);
            mbar_wait(done, 0, nullptr);
        }
    } else {
        // ---------------- epilogue: one thread per node and half ----------------
        // warps 2..9: lane quarter q = warp % 4 (the TMEM lanes this warp may
        // read), half h: the even or odd 32-column chunks of every tile
        const int e = warp - 2;
        const int q = warp & 3, h = e >> 2;   // lane quarter, group
        const int row = q * 32 + lane;
        const int node = tile_m * BM + row;
        const bool live = node < a.n_nodes;
        float nscale = 1.f, nbias = 0.f;
        unsigned nseed = 0;
        int box[6] = {0, 0, 0, 0, 0, 0};
        if (live) {
            if (a.node_scale) nscale = a.node_scale[node];
            if (a.node_bias) nbias = a.node_bias[node];
            nseed = a.node_seed ? a.node_seed[node] : 0u;
#pragma unroll
            for (int d = 0; d < 6; ++d) box[d] = a.node_box[node * 6 + d];
        }
        // this half's W best keys in registers, ascending (rk[0] the minimum);
        // keys start at 0, below every real key (ordered() of a score is > 0)
        unsigned long long rk[W];
        unsigned rp[W];
#pragma unroll
        for (int f = 0; f < W; ++f) {
            rk[f] = 0ull;
            rp[f] = 0xFFFFFFFFu;
        }
        unsigned long long root = 0ull;
        float thr = -INFINITY;
        unsigned g_seen = 0u;   // largest value of the shared bound this thread has read or published
        int i = 0;
        for (long long t = t_begin; t < t_end; ++t, ++i) {
            const int b = i & 1;
            const unsigned tph = (unsigned)(i >> 1) & 1u;
            bool ok = mbar_wait(&tfull[b], tph, &abort_s);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) {
                if (lane == 0) {
                    atomicExch(a.status, DEV_TC_WAIT);
                    abort_s = 1;
                }
                break;
            }
            tc_fence_after();
            const int pos0 = (int)(t * BN);
            const float s = nscale * (a.pos_scale ? __ldg(a.pos_scale + t) : 1.f);
            if (live && a.node_thr) {
                const unsigned g = *(volatile unsigned *)(a.node_thr + node);
                g_seen = g > g_seen ? g : g_seen;
                if (g) thr = fmaxf(thr, unordered(g));
            }
            // TI coordinates of the tile's first position
            const int x0 = pos0 % a.X, y0 = (pos0 / a.X) % a.Y, z0 = pos0 / (a.X * a.Y);
#pragma unroll 1
            for (int c = h; c < BN / 32; c += G) {
                float v[32];
                tmem_ld32(tmem + ((unsigned)(q * 32) << 16) + (unsigned)(b * BN + c * 32), v);
                // candidates of this lane (0 for a dead row, a chunk whose best
                // score is below the threshold, or no valid position); every
                // lane reaches the warp-wide round count below
                unsigned cand = 0u;
                const int pc = pos0 + c * 32;
                // a chunk's best score is exactly fmaf(max v, s, bias): fmaf is
                // monotone in v for s > 0
                float m01 = fmaxf(v[0], v[1]);
#pragma unroll
                for (int j = 2; j < 32; ++j) m01 = fmaxf(m01, v[j]);
                if (live && fmaf(m01, s, nbias) >= thr) {
                    // validity of the chunk's 32 positions for this node (its
                    // template inside the TI): the box cut row by row
                    unsigned vmask = 0u;
                    int x = x0 + c * 32, y = y0, z = z0;
                    while (x >= a.X) {
                        x -= a.X;
                        if (++y == a.Y) {
                            y = 0;
                            ++z;
                        }
                    }
                    const int end = (int)min((long long)pc + 32, a.n_pos);
                    int qp = pc;
                    while (qp < end) {
                        const int row0 = qp - x;
                        const int seg_end = min(end, row0 + a.X);
                        if (y >= box[2] && y < box[3] && z >= box[4] && z < box[5]) {
                            const int lo = max(qp, row0 + box[0]) - pc, hi = min(seg_end, row0 + box[1]) - pc;
                            if (lo < hi) vmask |= (hi >= 32 ? 0xFFFFFFFFu : ((1u << hi) - 1u)) & ~((1u << lo) - 1u);
                        }
                        qp = seg_end;
                        x = 0;
                        if (++y == a.Y) {
                            y = 0;
                            ++z;
                        }
                    }
                    // at least the threshold; a tie with the heap's own minimum
                    // qualifies only with a larger tie hash
                    const float thr_loc = root ? unordered((unsigned)(root >> 32)) : -INFINITY;
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const float sc = fmaf(v[j], s, nbias);
                        bool cj = sc >= thr && ((vmask >> j) & 1u);
                        if (cj && root != 0ull && sc == thr_loc) cj = tie_hash(nseed, (unsigned)(pc + j)) > (unsigned)root;
                        cand |= cj ? (1u << j) : 0u;
                    }
                }
                // insert them in rounds: every lane its next candidate
                const int rounds = __reduce_max_sync(0xffffffffu, __popc(cand));
                for (int r = 0; r < rounds; ++r) {
                    if (!cand) continue;
                    const int j = __ffs(cand) - 1;
                    cand &= cand - 1u;
                    // v[j] by a 5-level select tree
                    float t16[16], t8[8], t4[4], t2[2];
#pragma unroll
                    for (int u = 0; u < 16; ++u) t16[u] = (j & 1) ? v[2 * u + 1] : v[2 * u];
#pragma unroll
                    for (int u = 0; u < 8; ++u) t8[u] = (j & 2) ? t16[2 * u + 1] : t16[2 * u];
#pragma unroll
                    for (int u = 0; u < 4; ++u) t4[u] = (j & 4) ? t8[2 * u + 1] : t8[2 * u];
#pragma unroll
                    for (int u = 0; u < 2; ++u) t2[u] = (j & 8) ? t4[2 * u + 1] : t4[2 * u];
                    const float sc = fmaf((j & 16) ? t2[1] : t2[0], s, nbias);
                    const int p = pc + j;
                    const unsigned long long key = ((unsigned long long)ordered(sc) << 32) | tie_hash(nseed, (unsigned)p);
                    if (key <= root) continue;
                    sorted_insert<W>(rk, rp, key, (unsigned)p);
                    root = rk[0];
                    thr = root ? fmaxf(thr, unordered((unsigned)(root >> 32))) : thr;
                }
            }
            // publish this heap's minimum: a lower bound of the node's W-th best
            // over all positions, which every range may filter against.  The
            // bound only grows, so a minimum at or below the value last read
            // changes nothing: skipping it spares the bound's few cache lines,
            // which every CTA of the launch reads and updates, most updates
            if (live && root && a.node_thr && (unsigned)(root >> 32) > g_seen) {
                atomicMax(a.node_thr + node, (unsigned)(root >> 32));
                g_seen = (unsigned)(root >> 32);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[b]);
        }
        // the other groups hand their W best to group 0, which merges and
        // writes the node's W best of this range
        if (h > 0) {
#pragma unroll
            for (int f = 0; f < W; ++f) {
                hk[((h - 1) * W + f) * BM + row] = rk[f];
                hp[((h - 1) * W + f) * BM + row] = rp[f];
            }
        }
        asm volatile("bar.sync 1, %0;" ::"r"(EPI_WARPS * 32) : "memory");
        if (h == 0 && live) {
            for (int f = 0; f < (G - 1) * W; ++f) {
                const unsigned long long key = hk[f * BM + row];
                if (key > rk[0]) sorted_insert<W>(rk, rp, key, hp[f * BM + row]);
            }
            const size_t o = ((size_t)node * a.ranges + range) * W;
#pragma unroll
            for (int f = 0; f < W; ++f) {
                a.out_key[o + f] = rk[f];
                a.out_pos[o + f] = rp[f];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
}

// General BF16 GEMM on the tensor cores (the learned proposal's encoder):
// C[M x N] = A[M x K] * B[N x K]^T (+ bias[n]), A and B BF16 K-major with
// rows padded to the tile and K to 64 elements (zeros), C FP32 row-major.
// One 128 x BNG output tile per CTA: warp 0 streams the K blocks of A and B
// through a 4-stage ring with TMA, warp 1 allocates BNG TMEM columns and
// issues the MMAs (kind::f16, BF16 in, FP32 accumulate), warps 2-5 read the
// accumulator (one row per thread) and store the rows inside M x N.  Waits
// are bounded as in k_tc_shortlist.
template <int BNG>
__global__ void __launch_bounds__(192, 1)
    k_tc_gemm(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, TcGemmArgs g) {
    constexpr int STAGES = 4;
    constexpr int AB = BM * BKB, BB = BNG * BKB;
    extern __shared__ uint8_t smem_raw[];
    const unsigned raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *sA = smem, *sB = smem + STAGES * AB;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + STAGES * (AB + BB));
    uint64_t *full = bar, *empty = bar + STAGES, *tfull = bar + 2 * STAGES, *done = tfull + 1;
    __shared__ unsigned tmem_base_s;
    __shared__ volatile int abort_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile_m = blockIdx.x, tile_n = blockIdx.y;
    const int nkb = g.kpad / (BKB / 2);
    if (threadIdx.x == 0) {
        for (int i = 0; i < STAGES; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(tfull, 1);
        mbar_init(done, 1);
        abort_s = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                     "r"(BNG)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = tmem_base_s;
    if (warp == 0) {
        if (lane == 0) {
            int s = 0;
            unsigned ph = 0, issued_ph[STAGES];
            bool pending[STAGES];
            for (int i = 0; i < STAGES; ++i) pending[i] = false;
            bool ok = true;
            for (int kb = 0; kb < nkb; ++kb) {
                if (!mbar_wait(&empty[s], ph ^ 1u, &abort_s)) {
                    ok = false;
                    break;
                }
                mbar_expect_tx(&full[s], AB + BB);
                tma_load_2d(sA + s * AB, &map_a, &full[s], kb * (BKB / 2), tile_m * BM);
                tma_load_2d(sB + s * BB, &map_b, &full[s], kb * (BKB / 2), tile_n * BNG);
                pending[s] = true;
                issued_ph[s] = ph;
                if (++s == STAGES) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            if (!ok) {
                atomicExch(g.status, DEV_TC_WAIT);
                abort_s = 1;
            }
            for (int i = 0; i < STAGES; ++i)
                if (pending[i]) mbar_wait(&full[i], issued_ph[i], nullptr);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr unsigned idesc = make_idesc(1u, BM, BNG);
            int s = 0;
            unsigned ph = 0;
            bool ok = true;
            for (int kb = 0; kb < nkb; ++kb) {
                if (!mbar_wait(&full[s], ph, &abort_s)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint64_t ad = sw128_desc(smem_u32(sA + s * AB));
                const uint64_t bd = sw128_desc(smem_u32(sB + s * BB));
#pragma unroll
                for (int k = 0; k < 4; ++k) mma<0>(tmem, ad + (uint64_t)(2 * k), bd + (uint64_t)(2 * k), idesc, (kb | k) != 0);
                mma_commit(&empty[s]);
                if (++s == STAGES) {
                    s = 0;
                    ph ^= 1u;
                }
            }
            if (ok) {
                mma_commit(tfull);
            } else {
                atomicExch(g.status, DEV_TC_WAIT);
                abort_s = 1;
            }
            mma_commit(done);
            mbar_wait(done, 0, nullptr);
        }
    } else {
        const int q = warp & 3;   // the TMEM lane quarter this warp may read
        // the TMEM loads below are warp-collective: every lane takes the same branch
        const bool ok = __all_sync(0xffffffffu, mbar_wait(tfull, 0, &abort_s));
        if (ok) {
            tc_fence_after();
            const int row = tile_m * BM + q * 32 + lane;
            float v[32];
#pragma unroll 1
            for (int c = 0; c < BNG / 32; ++c) {
                tmem_ld32(tmem + ((unsigned)(q * 32) << 16) + (unsigned)(c * 32), v);
                if (row < g.M) {
                    float *crow = g.C + (long long)row * g.ldc;
                    const int col0 = tile_n * BNG + c * 32;
#pragma unroll
                    for (int i = 0; i < 32; ++i)
                        if (col0 + i < g.N) crow[col0 + i] = v[i] + (g.bias ? g.bias[col0 + i] : 0.f);
                }
            }
        } else if (lane == 0) {
            atomicExch(g.status, DEV_TC_WAIT);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BNG) : "memory");
    }
}

}  // namespace tc

// ---------------------------------------------------------------------------
// host side: tensor maps and launch
// ---------------------------------------------------------------------------
namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// rows x k_elems operand, row-major (K contiguous), element of `elem` bytes,
// boxes of one 128-byte K block x box_rows rows, 128-byte swizzle
cudaError_t make_map(CUtensorMap *m, const void *base, int elem, long long k_elems, long long rows, int box_rows) {
    auto enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    cuuint64_t dims[2] = {(cuuint64_t)k_elems, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(k_elems * elem)};
    cuuint32_t box[2] = {(cuuint32_t)(tc::BKB / elem), (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, elem == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_UINT8, 2,
                     const_cast<void *>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int KIND, int W>
cudaError_t launch_w(const CUtensorMap &ma, const CUtensorMap &mp, const TcArgs &a, int node_tiles,
                     cudaStream_t st) {
    constexpr int HEAP = (tc::epi_groups(W) - 1) * W * tc::BM * 12;
    constexpr int STAGES = 3;
    constexpr int SMEM = 1024 + STAGES * tc::STAGE_BYTES + HEAP + (2 * STAGES + 5) * 8;
    static_assert(SMEM <= 232448, "shared memory");
    auto kern = tc::k_tc_shortlist<KIND, W, STAGES>;
    // the shared-memory limit, once per device for this instantiation
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 0 || dev >= 64 || !done[dev]) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) done[dev] = true;
        }
    }
    dim3 grid((unsigned)node_tiles, (unsigned)a.ranges);
    return launch_pdl(kern, grid, dim3(tc::threads_for(W)), SMEM, st, ma, mp, a);
}

}  // namespace

int tc_supported_width(int w) { return w == 8 || w == 16 || w == 32; }

cudaError_t launch_tc_shortlist(int kind, int W, const void *a_mat, long long a_rows, const void *p_mat,
                                long long p_rows, long long k_elems, const TcArgs &args, cudaStream_t st) {
    const int elem = kind == 0 ? 2 : 1;
    if ((k_elems * elem) % tc::BKB != 0) return cudaErrorInvalidValue;
    if (a_rows % tc::BM != 0 || p_rows % tc::BN != 0) return cudaErrorInvalidValue;
    CUtensorMap ma, mp;
    cudaError_t e;
    if ((e = make_map(&ma, a_mat, elem, k_elems, a_rows, tc::BM)) != cudaSuccess) return e;
    if ((e = make_map(&mp, p_mat, elem, k_elems, p_rows, tc::BN)) != cudaSuccess) return e;
    TcArgs a = args;
    a.k_per_block = tc::BKB / elem;
    const int node_tiles = (int)(a_rows / tc::BM);
    if (kind == 0) {
        if (W == 8) return launch_w<0, 8>(ma, mp, a, node_tiles, st);
        if (W == 16) return launch_w<0, 16>(ma, mp, a, node_tiles, st);
        if (W == 32) return launch_w<0, 32>(ma, mp, a, node_tiles, st);
    } else {
        if (W == 8) return launch_w<1, 8>(ma, mp, a, node_tiles, st);
        if (W == 16) return launch_w<1, 16>(ma, mp, a, node_tiles, st);
        if (W == 32) return launch_w<1, 32>(ma, mp, a, node_tiles, st);
    }
    return cudaErrorInvalidValue;
}

namespace {
template <int BNG>
cudaError_t launch_gemm_bn(const CUtensorMap &ma, const CUtensorMap &mb, const TcGemmArgs &g, cudaStream_t st) {
    // alignment slack, the 4-stage ring, 10 mbarriers
    constexpr int SMEM = 1024 + 4 * (tc::BM + BNG) * tc::BKB + 10 * 8;
    static_assert(SMEM <= 232448, "shared memory");
    auto kern = tc::k_tc_gemm<BNG>;
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 0 || dev >= 64 || !done[dev]) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
            if (e != cudaSuccess) return e;
            if (dev >= 0 && dev < 64) done[dev] = true;
        }
    }
    dim3 grid((unsigned)((g.M + tc::BM - 1) / tc::BM), (unsigned)((g.N + BNG - 1) / BNG));
    kern<<<grid, 192, SMEM, st>>>(ma, mb, g);
    return cudaGetLastError();
}
}  // namespace

int tc_gemm_bn(int N) { return N <= 64 ? 64 : N <= 128 ? 128 : 256; }

cudaError_t launch_tc_gemm(const void *a_bf16, long long a_rows, const void *b_bf16, long long b_rows,
                           const TcGemmArgs &g, cudaStream_t st) {
    if (g.M <= 0 || g.N <= 0) return cudaSuccess;
    const int BNG = tc_gemm_bn(g.N);
    // operands are padded: rows to the tile, K to whole 64-element blocks
    if (g.kpad <= 0 || g.kpad % 64 || a_rows % tc::BM || b_rows % BNG || a_rows < g.M || b_rows < g.N)
        return cudaErrorInvalidValue;
    CUtensorMap ma, mb;
    cudaError_t e;
    if ((e = make_map(&ma, a_bf16, 2, g.kpad, a_rows, tc::BM)) != cudaSuccess) return e;
    if ((e = make_map(&mb, b_bf16, 2, g.kpad, b_rows, BNG)) != cudaSuccess) return e;
    if (BNG == 64) return launch_gemm_bn<64>(ma, mb, g, st);
    if (BNG == 128) return launch_gemm_bn<128>(ma, mb, g, st);
    return launch_gemm_bn<256>(ma, mb, g, st);
}

}  // namespace qsk

// ===========================================================================
// The tensor-core form inside the batched simulation
// ===========================================================================
#include "qsk_tc_nodes.cuh"

namespace qsk {
namespace {

// value of layer `ly` of the pattern matrix at TI cell q (natural index, x fastest)
__device__ __forceinline__ float layer_value(const float *__restrict__ ti, int nvar, long long q, const TcLayer &ly) {
    const float t = ti[q * nvar + ly.var];
    if (ly.kind == 0) return isnan(t) ? 0.f : t * t;
    if (ly.kind == 1) return isnan(t) ? 0.f : t;
    return t == ly.code ? 1.f : 0.f;
}

// P[p][j * L + l] = layer l at TI cell p + o_j (0 outside the TI); one warp
// per row.  FP8: pass 0 writes every row's largest magnitude to rowmax,
// k_tc_tile_scale turns each tile of 256 rows into one power-of-two scale
// (pos_scale[tile]), pass 1 writes the rows divided by their tile's scale.
__global__ void k_tc_pattern(TcPatternArgs A, int pass, float *__restrict__ rowmax) {
    const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int nd = A.nd;
    for (long long p = warp; p < A.rows; p += nwarps) {
        int pc[QSK_MAXD] = {0, 0, 0, 0};
        long long r = p;
        for (int d = 0; d < nd; ++d) {
            pc[d] = int(r % A.src[d]);
            r /= A.src[d];
        }
        const bool live = p < A.N;
        float scale = 1.f;
        if (A.fmt == 1 && pass == 0) {
            float mx = 0.f;
            if (live)
                for (long long k = lane; k < (long long)A.T * A.L; k += 32) {
                    const int j = int(k / A.L), l = int(k % A.L);
                    long long q = 0, st = 1;
                    bool in = true;
                    for (int d = 0; d < nd; ++d) {
                        const int c = pc[d] + A.tpl[j * nd + d];
                        in &= c >= 0 && c < A.src[d];
                        q += (long long)c * st;
                        st *= A.src[d];
                    }
                    if (in) mx = fmaxf(mx, fabsf(layer_value(A.ti, A.nvar, q, A.layer[l])));
                }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            if (lane == 0) rowmax[p] = mx;
            continue;
        }
        if (A.fmt == 1) scale = A.pos_scale[p >> 8];
        const float inv = 1.f / scale;
        for (long long k = lane; k < A.Kp; k += 32) {
            float v = 0.f;
            if (live && k < (long long)A.T * A.L) {
                const int j = int(k / A.L), l = int(k % A.L);
                long long q = 0, st = 1;
                bool in = true;
                for (int d = 0; d < nd; ++d) {
                    const int c = pc[d] + A.tpl[j * nd + d];
                    in &= c >= 0 && c < A.src[d];
                    q += (long long)c * st;
                    st *= A.src[d];
                }
                if (in) v = layer_value(A.ti, A.nvar, q, A.layer[l]) * inv;
            }
            store_elem(A.P, p * A.Kp + k, v, A.fmt);
        }
    }
}

__global__ void k_tc_tile_scale(long long tiles, const float *__restrict__ rowmax, float *__restrict__ scale) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tiles) return;
    float mx = 0.f;
    for (int r = 0; r < 256; ++r) mx = fmaxf(mx, rowmax[t * 256 + r]);
    scale[t] = pow2_scale(mx);
}

// largest template index among a node's neighbours; -1 for nodes without a
// neighbour other than the centre (marginal draw: the plain path)
__global__ void k_tc_tmax(long long nodes, int n, const int *__restrict__ nb_count, const int *__restrict__ nb_tpl,
                          int *__restrict__ tmax) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const int c = nb_count[i];
    int m = -1;
    if (c >= 2)
        for (int j = 0; j < c; ++j) m = max(m, nb_tpl[i * n + j]);
    tmax[i] = m;
}

// one warp per tensor slot: the node's row of A (coefficients of its terms at
// their template columns), its validity box and tie seed
__global__ void k_tc_nodes(TcNodeArgs A) {
    griddep_wait();   // launched programmatically after k_prep_sim
    griddep_launch();
    tc_nodes_warp(A, int((blockIdx.x * blockDim.x + threadIdx.x) >> 5), int(threadIdx.x & 31));
}

// exact score of one candidate from its staged layer values xs[t] (term t's
// gathered value), in the plain map's term order (FP32, bit-identical to
// k_map_records) and in FP64; `scale` is the term scale
__device__ __forceinline__ void exact_score_staged(const Term *__restrict__ tm, int nt, const float *xs, float &s32,
                                                   double &s64, double &scale) {
    float acc = 0.f;
    double a64 = 0.0, sc = 0.0;
    for (int t = 0; t < nt; ++t) {
        const Term T = tm[t];
        const float x = xs[t];
        if (T.op == OP_SQLIN) {
            acc = __fmaf_rn(T.a, __fmul_rn(x, x), acc);
            acc = __fmaf_rn(T.b, x, acc);
            a64 += (double)T.a * ((double)x * (double)x) + (double)T.b * (double)x;
            sc += -(double)T.a * ((double)x * (double)x) + ((double)T.b * (double)T.b) / (-4.0 * (double)T.a);
        } else if (T.op == OP_EQ) {
            acc = (x == T.b) ? __fadd_rn(acc, T.a) : acc;
            a64 += (x == T.b) ? (double)T.a : 0.0;
            sc += (double)T.a;
        } else if (T.op == OP_LIN) {
            acc = __fmaf_rn(T.a, x, acc);
            a64 += (double)T.a * (double)x;
            sc += fabs((double)T.a * (double)x);
        }
    }
    s32 = acc;
    s64 = a64;
    scale = sc;
}

// exact score of one candidate at scan index m, in the plain map's term order
// (FP32, bit-identical to k_map_records) and in FP64; `scale` is the term
// scale sum w (v^2 + t^2) (continuous) / sum w (categorical)
__device__ __forceinline__ void exact_score(const Term *__restrict__ tm, int nt, const float *__restrict__ layers,
                                            long long m, float &s32, double &s64, double &scale) {
    float acc = 0.f;
    double a64 = 0.0, sc = 0.0;
    for (int t = 0; t < nt; ++t) {
        const Term T = tm[t];
        const float x = __ldg(layers + T.base + m);
        if (T.op == OP_SQLIN) {
            acc = __fmaf_rn(T.a, __fmul_rn(x, x), acc);
            acc = __fmaf_rn(T.b, x, acc);
            a64 += (double)T.a * ((double)x * (double)x) + (double)T.b * (double)x;
            sc += -(double)T.a * ((double)x * (double)x) + ((double)T.b * (double)T.b) / (-4.0 * (double)T.a);
        } else if (T.op == OP_EQ) {
            acc = (x == T.b) ? __fadd_rn(acc, T.a) : acc;
            a64 += (x == T.b) ? (double)T.a : 0.0;
            sc += (double)T.a;
        } else if (T.op == OP_LIN) {
            acc = __fmaf_rn(T.a, x, acc);
            a64 += (double)T.a * (double)x;
            sc += fabs((double)T.a * (double)x);
        }
    }
    s32 = acc;
    s64 = a64;
    scale = sc;
}

constexpr int SEL_WARPS = 4;
constexpr int SEL_CAND = 768;    // candidates per slot staged in shared memory
constexpr int SEL_CPL = 8;       // shortlist entries per lane: at most 256 re-scored

// one warp per tensor slot: the S best candidates by approximate key, their
// exact scores, the node's k best by exact score (ties by the key's hash),
// the draw and the write-back
__global__ void __launch_bounds__(32 * SEL_WARPS) k_tc_select(TcSelectArgs A) {
    __shared__ unsigned long long skey[SEL_WARPS][SEL_CAND];
    __shared__ unsigned spos[SEL_WARPS][SEL_CAND];
    __shared__ Term sterm[SEL_WARPS][96];
    griddep_wait();   // launched programmatically after the shortlist
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * SEL_WARPS + w;
    if (b >= A.nslots) return;
    const Slot s = A.slots[b];
    const Geom &g = A.g;
    const int nt = s.nterms;
    const Term *tm = A.terms + (long long)b * A.maxterms;
    const bool small = nt <= 96;
    if (small)
        for (int t = lane; t < nt; t += 32) sterm[w][t] = tm[t];
    const int nc = A.ncand;
    // largest key a position outside the final shortlist can have by the
    // proposal (learned mode): the best of the ranges' heap minima (a full
    // heap's minimum bounds what that range left out)
    unsigned long long lout = 0ull;
    for (int c = lane; c < nc; c += 32) {
        const unsigned long long k = A.cand_key[(long long)b * nc + c];
        skey[w][c] = k;
        spos[w][c] = A.cand_pos[(long long)b * nc + c];
    }
    __syncwarp();
    if (A.fallback && A.conf_z > 0.f && A.range_w > 0) {
        for (int r = lane; r * A.range_w < nc; r += 32) {
            unsigned long long mn = ~0ull;
            for (int f = 0; f < A.range_w; ++f) mn = min(mn, skey[w][r * A.range_w + f]);
            lout = max(lout, mn);   // 0 when the range's heap was not full: it left nothing out
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lout = max(lout, __shfl_xor_sync(0xffffffffu, lout, o));
    }
    const Term *tt = small ? sterm[w] : tm;
    // the S largest keys (S rounds of warp argmax); lane r keeps round r and r+32
    unsigned long long mykey[SEL_CPL];
    unsigned mypos[SEL_CPL];
#pragma unroll
    for (int h = 0; h < SEL_CPL; ++h) {
        mykey[h] = 0ull;
        mypos[h] = 0u;
    }
    int nsel = 0;
    for (int r = 0; r < A.S; ++r) {
        unsigned long long bk = 0ull;
        int bi = -1;
        for (int c = lane; c < nc; c += 32) {
            const unsigned long long k = skey[w][c];
            if (k > bk) {
                bk = k;
                bi = c;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long ok = __shfl_xor_sync(0xffffffffu, bk, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ok > bk || (ok == bk && oi > bi)) {
                bk = ok;
                bi = oi;
            }
        }
        if (bk == 0ull) break;
        if (lane == (r & 31)) {
#pragma unroll
            for (int h = 0; h < SEL_CPL; ++h)
                if (h == (r >> 5)) {
                    mykey[h] = bk;
                    mypos[h] = spos[w][bi];
                }
        }
        __syncwarp();
        if (lane == 0) skey[w][bi] = 0ull;
        __syncwarp();
        ++nsel;
    }
    if (A.fallback && A.conf_z > 0.f) {
        unsigned long long nk = 0ull;
        for (int c = lane; c < nc; c += 32) nk = max(nk, skey[w][c]);   // best key not taken
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nk = max(nk, __shfl_xor_sync(0xffffffffu, nk, o));
        lout = max(lout, nk);
    }
    // exact scores of the shortlist: the scan index of every candidate, then
    // all (candidate, term) layer values gathered by the whole warp at once
    // into shared memory, then each candidate's term chain from there
    float e32[SEL_CPL];
    double e64[SEL_CPL], esc[SEL_CPL];
    unsigned hsh[SEL_CPL];
    bool live[SEL_CPL];
#pragma unroll
    for (int h = 0; h < SEL_CPL; ++h) {
        e32[h] = -INFINITY;
        e64[h] = -INFINITY;
        esc[h] = 0.0;
        hsh[h] = 0u;
        live[h] = false;
    }
    float errmax = 0.f;
    double errsum = 0.0;
    int errn = 0;
    int *msc = reinterpret_cast<int *>(&spos[w][0]);   // candidate list no longer needed
    for (int h = 0; h < SEL_CPL; ++h) {
        const int r = h * 32 + lane;
        if (r >= nsel) continue;
        // natural cell -> scan index of the reference's flipped space (cvtPositionToIndex)
        long long m = 0;
        unsigned rem = mypos[h];
        for (int d = 0; d < g.nd; ++d) {
            const int pd = int(rem % (unsigned)g.src[d]);
            rem /= (unsigned)g.src[d];
            m += (long long)(g.fft[d] - 1 - pd - s.mn[d]) * g.sstride[d];
        }
        msc[r] = (int)m;
    }
    __syncwarp();
    float *xs = reinterpret_cast<float *>(&skey[w][0]);   // 2 * SEL_CAND floats
    const int per = (small && nt > 0) ? max(1, min(nsel, (2 * SEL_CAND) / nt)) : 0;
    if (per > 0) {
        for (int r0 = 0; r0 < nsel; r0 += per) {
            const int r1 = min(nsel, r0 + per);
            for (int r = r0; r < r1; ++r) {
                const long long m = msc[r];
                for (int t = lane; t < nt; t += 32) xs[(r - r0) * nt + t] = __ldg(A.layers + tt[t].base + m);
            }
            __syncwarp();
            for (int h = 0; h < SEL_CPL; ++h) {
                const int r = h * 32 + lane;
                if (r >= r0 && r < r1) exact_score_staged(tt, nt, xs + (r - r0) * nt, e32[h], e64[h], esc[h]);
            }
            __syncwarp();
        }
    } else {
        for (int h = 0; h < SEL_CPL; ++h) {
            const int r = h * 32 + lane;
            if (r < nsel) exact_score(tt, nt, A.layers, (long long)msc[r], e32[h], e64[h], esc[h]);
        }
    }
    for (int h = 0; h < SEL_CPL; ++h) {
        const int r = h * 32 + lane;
        if (r >= nsel) continue;
        const float approx = tc::unordered((unsigned)(mykey[h] >> 32));
        const double err = fabs((double)approx - e64[h]) / (esc[h] > 0.0 ? esc[h] : 1.0);
        errmax = fmaxf(errmax, (float)err);
        errsum += err;
        ++errn;
        hsh[h] = (unsigned)(mykey[h] & 0xFFFFFFFFull);
        live[h] = true;
    }
    // the node's K best by exact score (FP64 or FP32; equal scores ordered by
    // the candidate's tie hash), extracted in descending order; the draw takes
    // rank sel (the quantile rank of sample(), quantileSamplingModule.hpp:113)
    const int K = s.K;
    unsigned chosen = 0xFFFFFFFFu;
    float chosen32 = -INFINITY;
    double chosen_sc = 0.0;
    const bool f64 = A.fp64 != 0;
    double kth_score = -INFINITY;   // the K-th best exact score (ranking precision)
    for (int k = 0; k < K && k < nsel; ++k) {
        int bh = -1;
        for (int h = 0; h < SEL_CPL; ++h) {
            if (!live[h]) continue;
            if (bh < 0) {
                bh = h;
                continue;
            }
            const bool better = f64 ? (e64[h] > e64[bh] || (e64[h] == e64[bh] && hsh[h] > hsh[bh]))
                                    : (e32[h] > e32[bh] || (e32[h] == e32[bh] && hsh[h] > hsh[bh]));
            if (better) bh = h;
        }
        double bv = bh >= 0 ? (f64 ? e64[bh] : (double)e32[bh]) : -INFINITY;
        unsigned bhs = bh >= 0 ? hsh[bh] : 0u;
        int bl = bh >= 0 ? lane : -1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const unsigned oh = __shfl_xor_sync(0xffffffffu, bhs, o);
            const int ol = __shfl_xor_sync(0xffffffffu, bl, o);
            if (ol >= 0 && (bl < 0 || ov > bv || (ov == bv && (oh > bhs || (oh == bhs && ol > bl))))) {
                bv = ov;
                bhs = oh;
                bl = ol;
            }
        }
        if (bl < 0) break;
        const int wh = __shfl_sync(0xffffffffu, bh, bl);
        unsigned wp0 = 0u;
        float w320 = 0.f;
        double wsc0 = 0.0;
#pragma unroll
        for (int h = 0; h < SEL_CPL; ++h)
            if (h == wh) {
                wp0 = mypos[h];
                w320 = e32[h];
                wsc0 = esc[h];
                if (lane == bl) live[h] = false;
            }
        const unsigned wp = __shfl_sync(0xffffffffu, wp0, bl);
        const float w32 = __shfl_sync(0xffffffffu, w320, bl);
        const double wsc = __shfl_sync(0xffffffffu, wsc0, bl);
        // rank sel, or the last one found when fewer than sel + 1 exist
        if (k <= s.sel) {
            chosen = wp;
            chosen32 = w32;
            chosen_sc = wsc;
        }
        kth_score = bv;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        errmax = fmaxf(errmax, __shfl_xor_sync(0xffffffffu, errmax, o));
        errsum += __shfl_xor_sync(0xffffffffu, errsum, o);
        errn += __shfl_xor_sync(0xffffffffu, errn, o);
    }
    // confidence (learned proposal): the exact best of the shortlist must rank
    // among its first conf_rank by the proposal's own score; otherwise the
    // node goes to the exact map (no write-back here)
    bool confident = true;
    if (A.fallback) {
        int br = 0x7FFFFFFF;
        double bv2 = -INFINITY;
        unsigned bh2 = 0u;
        for (int h = 0; h < SEL_CPL; ++h) {
            const int r = h * 32 + lane;
            if (r >= nsel) continue;
            const double v2 = f64 ? e64[h] : (double)e32[h];
            if (v2 > bv2 || (v2 == bv2 && hsh[h] > bh2)) {
                bv2 = v2;
                bh2 = hsh[h];
                br = r;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv2, o);
            const unsigned oh = __shfl_xor_sync(0xffffffffu, bh2, o);
            const int orr = __shfl_xor_sync(0xffffffffu, br, o);
            if (ov > bv2 || (ov == bv2 && (oh > bh2 || (oh == bh2 && orr < br)))) {
                bv2 = ov;
                bh2 = oh;
                br = orr;
            }
        }
        confident = nsel > 0 && br < A.conf_rank;
        if (A.conf_z > 0.f) {
            // exact score against proposal score over the shortlist: s = a L + b
            // with residual sd; a position left out has L <= L_out, so its
            // score is below a L_out + b + z sd with high probability; the
            // node is confident when its k-th best exact score clears that
            double n = 0, sl = 0, ss = 0, sll = 0, sls = 0;
            for (int h = 0; h < SEL_CPL; ++h) {
                const int r = h * 32 + lane;
                if (r >= nsel) continue;
                const double L = (double)tc::unordered((unsigned)(mykey[h] >> 32));
                const double v2 = f64 ? e64[h] : (double)e32[h];
                n += 1;
                sl += L;
                ss += v2;
                sll += L * L;
                sls += L * v2;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                n += __shfl_xor_sync(0xffffffffu, n, o);
                sl += __shfl_xor_sync(0xffffffffu, sl, o);
                ss += __shfl_xor_sync(0xffffffffu, ss, o);
                sll += __shfl_xor_sync(0xffffffffu, sll, o);
                sls += __shfl_xor_sync(0xffffffffu, sls, o);
            }
            const double den = n * sll - sl * sl;
            const double aa = den > 0 ? (n * sls - sl * ss) / den : 0.0;
            const double bb = n > 0 ? (ss - aa * sl) / n : 0.0;
            double r2 = 0;
            for (int h = 0; h < SEL_CPL; ++h) {
                const int r = h * 32 + lane;
                if (r >= nsel) continue;
                const double L = (double)tc::unordered((unsigned)(mykey[h] >> 32));
                const double v2 = f64 ? e64[h] : (double)e32[h];
                const double d = v2 - aa * L - bb;
                r2 += d * d;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) r2 += __shfl_xor_sync(0xffffffffu, r2, o);
            const double sd = n > 1 ? sqrt(r2 / n) : 0.0;
            // variance of the exact scores: the fit must explain at least
            // the fraction conf_r2 of it for its extrapolation to be trusted
            const double var = n > 1 ? 1.0 : 0.0;
            double tv = 0;
            for (int h = 0; h < SEL_CPL; ++h) {
                const int r = h * 32 + lane;
                if (r >= nsel) continue;
                const double v2 = (f64 ? e64[h] : (double)e32[h]) - (n > 0 ? ss / n : 0.0);
                tv += v2 * v2;
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) tv += __shfl_xor_sync(0xffffffffu, tv, o);
            const bool fits = var > 0 && tv > 0 && aa > 0 && r2 <= (1.0 - (double)A.conf_r2) * tv;
            const double Lout = lout ? (double)tc::unordered((unsigned)(lout >> 32)) : -INFINITY;
            const double bound = lout ? aa * Lout + bb + (double)A.conf_z * sd : -INFINITY;
            // the k-th best exact score of the shortlist (the K-th extraction)
            confident = nsel >= K && fits && kth_score >= bound;
        }
    }
    if (lane == 0) {
        if (A.err_max) atomicMax(A.err_max, __float_as_uint(errmax));
        if (A.err_sum) atomicAdd(A.err_sum, errsum);
        if (A.err_n) atomicAdd(A.err_n, (unsigned long long)errn);
        if (A.fallback) A.fallback[b] = confident ? 0 : 1;
        if (!confident) return;
        if (chosen == 0xFFFFFFFFu) {
            if (A.status) atomicExch(A.status, DEV_BAD_INDEX);
            return;
        }
        if (A.node_cell) A.node_cell[s.node] = chosen;
        if (A.drawn_score) A.drawn_score[s.node] = chosen32;
        if (A.drawn_scale) A.drawn_scale[s.node] = (float)chosen_sc;
        if (A.state)
            for (int v = 0; v < A.nvar; ++v) {
                float *dst = A.state + (long long)s.cell * A.nvar + v;
                if (isnan(*dst)) *dst = A.ti[(long long)chosen * A.nvar + v];
            }
        if (A.id_image) A.id_image[s.cell] = chosen * A.nti + A.ti_id;
    }
}

// regret audit: the plain path's exact k best of audited node a (values
// descending) against the candidate the tensor path drew for it
__global__ void k_tc_audit(int n, const int *__restrict__ nodes, int K, const float *__restrict__ plain_val,
                           const float *__restrict__ drawn_score, const float *__restrict__ drawn_scale, float tol,
                           unsigned long long *__restrict__ counts) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const int node = nodes[a];
    const float kth = plain_val[(long long)a * K + K - 1];
    const float d = drawn_score[node];
    const float t = tol * drawn_scale[node];
    unsigned long long c0 = 1, c1 = 0, c2 = 0;
    if (d < kth - t) c1 = 1;          // outside the exact k-best set
    else if (d < kth) c2 = 1;         // below the k-th by at most the near-tie tolerance
    atomicAdd(counts + 0, c0);
    atomicAdd(counts + 1, c1);
    atomicAdd(counts + 2, c2);
}

}  // namespace

cudaError_t launch_tc_pattern(const TcPatternArgs &a, float *rowmax, cudaStream_t st) {
    long long warps = a.rows;
    long long blocks = (warps * 32 + 255) / 256;
    if (blocks > 148LL * 64) blocks = 148LL * 64;
    if (a.fmt == 1) {
        k_tc_pattern<<<(unsigned)blocks, 256, 0, st>>>(a, 0, rowmax);
        const long long tiles = a.rows / 256;
        k_tc_tile_scale<<<(unsigned)((tiles + 255) / 256), 256, 0, st>>>(tiles, rowmax, a.pos_scale);
    }
    k_tc_pattern<<<(unsigned)blocks, 256, 0, st>>>(a, 1, rowmax);
    return cudaGetLastError();
}

cudaError_t launch_tc_tmax(long long nodes, int n, const int *nb_count, const int *nb_tpl, int *tmax, cudaStream_t st) {
    if (nodes <= 0) return cudaSuccess;
    k_tc_tmax<<<(unsigned)((nodes + 255) / 256), 256, 0, st>>>(nodes, n, nb_count, nb_tpl, tmax);
    return cudaGetLastError();
}

cudaError_t launch_tc_nodes(const TcNodeArgs &a, cudaStream_t st) {
    if (a.A && (a.rows < a.nslots || (a.Kp * (a.fmt == 1 ? 1 : 2)) % 16 != 0)) return cudaErrorInvalidValue;
    const long long warps = a.A ? a.rows : a.nslots;
    const long long blocks = (warps * 32 + 255) / 256;
    return launch_pdl(k_tc_nodes, dim3((unsigned)blocks), dim3(256), 0, st, a);
}

cudaError_t launch_tc_select(const TcSelectArgs &a, cudaStream_t st) {
    if (a.ncand > SEL_CAND || a.S > 32 * SEL_CPL) return cudaErrorInvalidValue;
    return launch_pdl(k_tc_select, dim3((unsigned)((a.nslots + SEL_WARPS - 1) / SEL_WARPS)), dim3(32 * SEL_WARPS), 0,
                      st, a);
}

cudaError_t launch_tc_audit(int n, const int *nodes, int K, const float *plain_val, const float *drawn_score,
                            const float *drawn_scale, float tol, unsigned long long *counts, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_tc_audit<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, nodes, K, plain_val, drawn_score, drawn_scale, tol, counts);
    return cudaGetLastError();
}

}  // namespace qsk

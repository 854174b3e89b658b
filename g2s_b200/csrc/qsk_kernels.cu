// CUDA kernels of the B200 QuickSampling (QS) hot path, sm_100a.
//
// Per batch of independent path nodes ("slots"):
//   k_prep_sim     neighbour values -> per-node term list, border bounds
//                  (G2S include/simulation.hpp:447-537, quantileSamplingModule.hpp:368-457,
//                   DataImage.hpp:626-710, CPUThreadDevice.cpp:352-366,454-477)
//   k_map_records  mismatch map of every scan position in FP32 (direct sum in
//                  the reference's layer decomposition, CPUThreadDevice.cpp:349-490)
//                  fused with a warp prefix-top-K filter that keeps only the
//                  positions that can enter the running k-best ("records")
//   k_replay       exact replay of the reference's k-biggest scan with its
//                  mt19937 reservoir tie-breaking (fKb.hpp:58-92,121-132,
//                  quantileSamplingModule.hpp:45-49,525-557) over the records,
//                  then the draw and the write-back (quantileSamplingModule.hpp:90-126,
//                  CPUThreadDevice.cpp:257-268, simulation.hpp:586-666)
//   k_map_bits     the same map for categorical patterns with unit weights,
//                  bit-sliced (one bit plane per category), same records
// Setup kernels: k_build_layers (DataImage.hpp:538-599), k_neighbours
// (simulation.hpp:447-511, run for every path node at once), k_level_flow /
// k_level_count / k_level_scatter (dependency levels of the path DAG, nodes
// grouped by level).
#include <cuda_runtime.h>

#include <atomic>
#include <math_constants.h>
#include <cstdint>

#include "qsk_internal.h"
#include "qsk_pdl.cuh"
#include "qsk_tc_nodes.cuh"

namespace qsk {

// ---------------------------------------------------------------------------
// small helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// merge two descending top-K lists (register arrays, static indices only):
// c_t = max_{i=0..t+1} min(a_{i-1}, b_{t-i}), with a_{-1} = b_{-1} = +inf.
template <int K>
__device__ __forceinline__ void topk_merge(const float (&a)[K], const float (&b)[K], float (&c)[K]) {
#pragma unroll
    for (int t = 0; t < K; ++t) {
        float best = -CUDART_INF_F;
#pragma unroll
        for (int i = 0; i <= t + 1; ++i) {
            float ai = (i == 0) ? CUDART_INF_F : a[i - 1];
            float bj = (t - i >= 0) ? b[t - i] : CUDART_INF_F;
            best = fmaxf(best, fminf(ai, bj));
        }
        c[t] = best;
    }
}

template <int KF>
__device__ __forceinline__ void topk_insert(float (&st)[KF], float x) {
    // insert x into the descending list st, dropping the smallest
#pragma unroll
    for (int s = KF - 1; s >= 0; --s) {
        float prev = (s > 0) ? st[s > 0 ? s - 1 : 0] : CUDART_INF_F;
        // new st[s] = max(min(prev, x), st[s])
        st[s] = fmaxf(st[s], fminf(prev, x));
    }
}

// number of valid scan positions < x (x in [0, N])
__device__ long long valid_prefix(const Geom &g, const int *lo, long long x) {
    long long vd[QSK_MAXD];
    long long acc = 1;
    for (int d = 0; d < g.nd; ++d) {
        vd[d] = acc;
        long long w = g.fft[d] - lo[d];
        acc *= (w > 0 ? w : 0);
    }
    if (x >= g.N) return acc;
    // scan indices are below 2^31 (int record indices): 32-bit digits
    long long count = 0;
    const unsigned ux = (unsigned)x;
    for (int d = g.nd - 1; d >= 0; --d) {
        const int digit = int((ux / (unsigned)g.sstride[d]) % (unsigned)g.fft[d]);
        const int t = digit - lo[d];
        if (t > 0) count += (long long)t * vd[d];
        if (digit < lo[d]) break;
    }
    return count;
}

// ---------------------------------------------------------------------------
// layers: flipped copy of each TI variable (DataImage.hpp:538-599)
// continuous: value with NaN -> 0 ; categorical: value kept as the category
// code (NaN stays NaN, so it never equals a code).  Positions of the fft grid
// outside the TI hold 0 (continuous) / NaN (categorical).
// ---------------------------------------------------------------------------
__global__ void k_build_layers(const float *__restrict__ ti, int nvar, const int *__restrict__ types, Geom g,
                               float *__restrict__ layers, int missing) {
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.N) return;
    // q is an fft-grid flat index of the flipped array: coord = fft-1-digit
    long long src_flat = 0, sstr = 1;
    bool inside = true;
    for (int d = 0; d < g.nd; ++d) {
        long long digit = (q / g.sstride[d]) % g.fft[d];
        long long c = g.fft[d] - 1 - digit;
        inside &= c < g.src[d];
        src_flat += c * sstr;
        sstr *= g.src[d];
    }
    for (int v = 0; v < nvar; ++v) {
        float x;
        if (inside) {
            x = ti[src_flat * nvar + v];
            if (types[v] == 0 && isnan(x) && !missing) x = 0.f;
        } else {
            x = types[v] == 0 ? 0.f : CUDART_NAN_F;
        }
        layers[(long long)v * g.N + q] = x;
    }
    if (missing) {
        // mask layer (DataImage.hpp:582-595): 1 where the TI cell is informed
        layers[(long long)nvar * g.N + q] = (inside && !isnan(ti[src_flat * nvar])) ? 1.f : 0.f;
    }
}

// ---------------------------------------------------------------------------
// neighbour search for every path node (simulation.hpp:447-511, single n,
// non-strict informed rule: cells with path order <= the node's, the node
// itself included).
// ---------------------------------------------------------------------------
// one warp per node: 32 template offsets tested per step, accepted ones
// appended in template order
__global__ void k_neighbours(GridDesc dg, const int *__restrict__ tpl, int ntpl, const unsigned *__restrict__ path,
                             unsigned begin, long long nodes, const unsigned *__restrict__ posterior, int n,
                             int *__restrict__ nb_count, int *__restrict__ nb_tpl, unsigned *__restrict__ nb_cell,
                             const int *__restrict__ node_kernel, const int *__restrict__ tpl_range,
                             const int *__restrict__ node_lim) {
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= nodes) return;
    const unsigned cell = path[begin + i];
    const unsigned order = posterior[cell];
    int c0[QSK_MAXD];
    long long rem = cell;
    for (int d = 0; d < dg.nd; ++d) {
        c0[d] = int(rem % dg.dims[d]);
        rem /= dg.dims[d];
    }
    // template of this node's kernel (-kii) and its neighbour limit (-n per variable / -ni)
    int tb = 0, tn = ntpl, lim = n;
    if (node_kernel) {
        const int q = node_kernel[i];
        tb = tpl_range[2 * q];
        tn = tpl_range[2 * q + 1];
    }
    if (node_lim) lim = min(node_lim[i], n);
    int cnt = 0;
    for (int t0 = 0; t0 < tn && cnt < lim; t0 += 32) {
        const int t = t0 + lane;
        bool acc = false;
        long long nc = 0;
        if (t < tn) {
            bool ok = true;
            for (int d = 0; d < dg.nd; ++d) {
                int c = c0[d] + tpl[(tb + t) * dg.nd + d];
                ok &= (c >= 0) && (c < dg.dims[d]);
                nc += (long long)c * dg.stride[d];
            }
            acc = ok && posterior[nc] <= order;
        }
        const unsigned bal = __ballot_sync(0xffffffffu, acc);
        const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
        if (acc && pos < lim) {
            nb_tpl[i * n + pos] = tb + t;
            nb_cell[i * n + pos] = unsigned(nc);
        }
        cnt += __popc(bal);
    }
    if (lane == 0) nb_count[i] = cnt < lim ? cnt : lim;
}

// -fs: one warp per (cell, variable) node.  A cell is taken when a variable
// that still needs neighbours was simulated there strictly before the node
// (posterior < order, simulation.hpp:822-872); the variables it contributes
// are recorded in nb_mask.  The 32 offsets of a step are tested in parallel,
// then taken in template order with the per-variable counts.
__global__ void k_neighbours_full(GridDesc dg, const int *__restrict__ tpl, int ntpl, const unsigned *__restrict__ path,
                                  unsigned begin, long long nodes, const unsigned *__restrict__ posterior, int nvar,
                                  int n, const int *__restrict__ node_nv, int *__restrict__ nb_count,
                                  int *__restrict__ nb_tpl, unsigned *__restrict__ nb_cell,
                                  unsigned char *__restrict__ nb_mask, const int *__restrict__ node_kernel,
                                  const int *__restrict__ tpl_range) {
    const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= nodes) return;
    const unsigned value = path[begin + i];
    const unsigned cell = value / unsigned(nvar);
    const unsigned order = posterior[value];
    int c0[QSK_MAXD];
    long long rem = cell;
    for (int d = 0; d < dg.nd; ++d) {
        c0[d] = int(rem % dg.dims[d]);
        rem /= dg.dims[d];
    }
    int tb = 0, tn = ntpl;
    if (node_kernel) {
        const int q = node_kernel[i];
        tb = tpl_range[2 * q];
        tn = tpl_range[2 * q + 1];
    }
    int need[4] = {0, 0, 0, 0};   // remaining count per variable
    unsigned needm = 0;
    for (int v = 0; v < nvar && v < 4; ++v) {
        need[v] = node_nv ? node_nv[i * nvar + v] : n;
        if (need[v] > 0) needm |= 1u << v;
    }
    int cnt = 0;
    for (int t0 = 0; t0 < tn && needm && cnt < n; t0 += 32) {
        const int t = t0 + lane;
        unsigned im = 0;
        long long nc = 0;
        if (t < tn) {
            bool ok = true;
            for (int d = 0; d < dg.nd; ++d) {
                int c = c0[d] + tpl[(tb + t) * dg.nd + d];
                ok &= (c >= 0) && (c < dg.dims[d]);
                nc += (long long)c * dg.stride[d];
            }
            if (ok)
                for (int v = 0; v < nvar && v < 4; ++v)
                    if (posterior[nc * nvar + v] < order) im |= 1u << v;
        }
        unsigned cand = __ballot_sync(0xffffffffu, (im & needm) != 0u);
        while (cand && needm && cnt < n) {
            const int l = __ffs(cand) - 1;
            cand &= cand - 1u;
            const unsigned m = __shfl_sync(0xffffffffu, im, l) & needm;
            if (!m) continue;
            if (lane == l) {
                nb_tpl[i * n + cnt] = tb + t;
                nb_cell[i * n + cnt] = unsigned(nc);
                nb_mask[i * n + cnt] = (unsigned char)m;
            }
            for (int v = 0; v < 4; ++v)
                if ((m >> v) & 1u && --need[v] == 0) needm &= ~(1u << v);
            ++cnt;
        }
    }
    if (lane == 0) nb_count[i] = cnt;
}

// ---------------------------------------------------------------------------
// dependency levels: level(i) = 1 + max level(j) over the node's informed
// neighbours j that are themselves path nodes (0 without any) -- the longest
// path to i in the path DAG (dependencies always point to smaller path
// indices).  One pass in path order (k_level_flow), then a counting sort of
// the nodes by level (k_level_count, the scan, k_level_scatter).
// ---------------------------------------------------------------------------
// dependency nodes of neighbour j of node i: the cell's node, or (-fs, with
// nb_mask) the nodes of the cell's values that the neighbour contributes
template <class F>
__device__ __forceinline__ void for_each_dep(long long i, int j, int n, const unsigned *__restrict__ nb_cell,
                                             const unsigned char *__restrict__ nb_mask, int nvar,
                                             const int *__restrict__ node_of, F f) {
    const unsigned c = nb_cell[i * n + j];
    if (!nb_mask) {
        const int d = node_of[c];
        if (d >= 0 && (long long)d != i) f(d);
        return;
    }
    const unsigned m = nb_mask[i * n + j];
    for (int v = 0; v < nvar; ++v)
        if ((m >> v) & 1u) {
            const int d = node_of[(long long)c * nvar + v];
            if (d >= 0 && (long long)d != i) f(d);
        }
}

// One warp per node, nodes taken in path order from a ticket.  A node's
// dependencies have smaller path indices, so they were taken earlier by warps
// that are running; the smallest unfinished node waits on finished nodes only,
// so every wait ends.  The waits are bounded all the same: past `spin_limit`
// polls of one dependency (2^22 by default, about a second with the back-off)
// the kernel records DEV_LEVEL_WAIT and moves on (the host then fails the
// run).  `hold` (normally -1) names a node whose level is never published:
// a host-side injection that makes its dependants' waits run out, so that the
// failure path can be exercised without a fault.
// The level words start at -1; a level is published with one volatile store
// and read with volatile loads (it carries no other data).
__global__ void k_level_flow(long long nodes, int n, const int *__restrict__ nb_count,
                             const unsigned *__restrict__ nb_cell, const unsigned char *__restrict__ nb_mask, int nvar,
                             const int *__restrict__ node_of, int *level, int *ticket, int *nl_out, int *status,
                             unsigned spin_limit, long long hold) {
    const int lane = threadIdx.x & 31;
    volatile int *vlevel = level;
    for (;;) {
        int i = 0;
        if (lane == 0) i = atomicAdd(ticket, 1);
        i = __shfl_sync(0xffffffffu, i, 0);
        if ((long long)i >= nodes) return;
        const int c = nb_count[i];
        int mx = -1;
        bool bad = false, late = false;
        for (int j = lane; j < c; j += 32)
            for_each_dep(i, j, n, nb_cell, nb_mask, nvar, node_of, [&](int d) {
                if (d >= i) {
                    bad = true;
                    return;
                }
                int lv = vlevel[d];
                unsigned spins = 0;
                while (lv < 0) {
                    if (++spins > spin_limit) {
                        late = true;
                        lv = 0;
                        break;
                    }
                    __nanosleep(128);
                    lv = vlevel[d];
                }
                mx = max(mx, lv);
            });
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, off));
        const bool any_bad = __any_sync(0xffffffffu, bad), any_late = __any_sync(0xffffffffu, late);
        if (lane == 0) {
            if (any_bad) atomicExch(status, DEV_BAD_INDEX);
            if (any_late) atomicExch(status, DEV_LEVEL_WAIT);
            if ((long long)i != hold) {
                vlevel[i] = mx + 1;
                atomicMax(nl_out, mx + 2);
            }
        }
    }
}

__global__ void k_level_count(long long nodes, const int *__restrict__ level, int *__restrict__ cnt) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nodes && level[i] >= 0) atomicAdd(&cnt[level[i]], 1);   // < 0: held back (the run fails)
}

// exclusive scan in three passes: 1024-element tiles, tile sums, add
__global__ void __launch_bounds__(1024) k_scan_tiles(long long count, const int *__restrict__ in, int *__restrict__ out,
                                                     int *__restrict__ tile_sum) {
    __shared__ int warp_sum[32];
    const long long i = (long long)blockIdx.x * 1024 + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int x = i < count ? in[i] : 0;
    int incl = x;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) warp_sum[w] = incl;
    __syncthreads();
    if (w == 0) {
        int ws = warp_sum[lane];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, ws, off);
            if (lane >= off) ws += y;
        }
        warp_sum[lane] = ws;   // inclusive
    }
    __syncthreads();
    const int base = w > 0 ? warp_sum[w - 1] : 0;
    if (i < count) out[i] = base + incl - x;
    if (threadIdx.x == 1023) tile_sum[blockIdx.x] = base + incl;
}

__global__ void k_scan_sums(int ntiles, int *__restrict__ tile_sum) {
    if (threadIdx.x == 0) {
        int s = 0;
        for (int t = 0; t < ntiles; ++t) {
            const int v = tile_sum[t];
            tile_sum[t] = s;
            s += v;
        }
        tile_sum[ntiles] = s;
    }
}

__global__ void k_scan_add(long long count, int *__restrict__ out, int *__restrict__ cursor,
                           const int *__restrict__ tile_sum) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) {
        const int v = out[i] + tile_sum[i / 1024];
        out[i] = v;
        cursor[i] = v;
    } else if (i == count) {
        const int v = tile_sum[(count + 1023) / 1024];
        out[i] = v;
    }
}

// nodes grouped by level (order inside a level is free: its nodes are independent)
__global__ void k_level_scatter(long long nodes, const int *__restrict__ level, int *__restrict__ cursor,
                                int *__restrict__ level_nodes) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nodes && level[i] >= 0) level_nodes[atomicAdd(&cursor[level[i]], 1)] = int(i);
}

// ---------------------------------------------------------------------------
// selected rank of the draw, exactly as compiled in the reference
// (quantileSamplingModule.hpp:113 with the double overloads of ceil/floor)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int selected_index(float seed, float k, unsigned nti) {
    double prod = (double)__fmul_rn(seed, k);
    double c = ceil((double)__fdiv_rn((float)nti, k));
    return int(floor(prod * (c / (double)nti)));
}

// ---------------------------------------------------------------------------
// prep for the simulation: one warp per slot
// ---------------------------------------------------------------------------
// The part of a node's slot that follows from the neighbour lists and the
// initial grid alone (not from simulated values), shared by k_prep_sim and
// k_mt_prep: candidate count, neighbour offset minima, first valid scan
// coordinate per dimension, number of valid positions, marginal draw.
struct NodeGeom {
    float lk;
    int Ki;
    int mn[QSK_MAXD];
    int lo[QSK_MAXD];
    long long nvalid;
    bool skip;
};

__device__ NodeGeom node_geometry(const SimPrepArgs &A, int i, unsigned cell, int lane) {
    NodeGeom r;
    const int cnt = A.nb_count[i];
    const int nd = A.g.nd;
    // candidate count of this node: -kvi or k (quantileSamplingModule.hpp:90-113)
    r.lk = A.node_k ? A.node_k[i] : A.k;
    int Ki = int(ceilf(r.lk));
    r.Ki = Ki < 1 ? 1 : (Ki > QSK_KMAX ? QSK_KMAX : Ki);
    // vector simulation: data at the centre also forces a search
    // (simulation.hpp:565-584); -fs draws from the marginal below two
    // neighbours (simulation.hpp:952-965)
    bool centreData = false;
    if (!A.full)
        for (int v = 0; v < A.nvar; ++v) centreData |= !isnan(A.init[(long long)cell * A.nvar + v]);
    // min / max of the neighbour offsets, starting from 0 (AcceleratorDevice.cpp:95-112)
    int mn[QSK_MAXD], mx[QSK_MAXD];
#pragma unroll
    for (int d = 0; d < QSK_MAXD; ++d) { mn[d] = 0; mx[d] = 0; }
    for (int j = lane; j < cnt; j += 32) {
        int t = A.nb_tpl[(long long)i * A.n + j];
        for (int d = 0; d < nd; ++d) {
            int o = A.tpl[t * nd + d];
            mn[d] = min(mn[d], o);
            mx[d] = max(mx[d], o);
        }
    }
#pragma unroll
    for (int d = 0; d < QSK_MAXD; ++d) {
        for (int off = 16; off > 0; off >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], off));
            mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], off));
        }
    }
    r.nvalid = 1;
    for (int d = 0; d < QSK_MAXD; ++d) {
        r.mn[d] = mn[d];
        int lo = 0;
        if (d < nd) {
            lo = A.g.fft[d] - (A.g.src[d] - (mx[d] - mn[d]));
            lo = lo < 0 ? 0 : (lo > A.g.fft[d] ? A.g.fft[d] : lo);
            r.nvalid *= (A.g.fft[d] - lo);
        }
        r.lo[d] = lo;
    }
    r.skip = cnt <= 1 && !centreData;   // marginal draw (simulation.hpp:586-605)
    return r;
}

// -nV: scan index of the TI cell that continues neighbour 1's source (cell
// id_src, template offset tpl1) (simulation.hpp:556-583,
// quantileSamplingModule.hpp:518-523), or -1 outside the scan
__device__ int verbatim_excl(const Geom &g, const int *tpl1, unsigned id_src, const int *mn) {
    const int nd = g.nd;
    unsigned src = id_src;
    long long pf = 0, st = 1;
    for (int d = 0; d < nd; ++d) {
        int dim = g.src[d];
        int c = int(src % (unsigned)dim) - tpl1[d];
        src /= (unsigned)dim;
        c = ((c % dim) + dim) % dim;
        pf += (long long)c * st;
        st *= dim;
    }
    // cvtPositionToIndex (CPUThreadDevice.cpp:270-284), unsigned arithmetic
    unsigned position = (unsigned)pf, index = 0, div = 1;
    for (int d = nd - 1; d >= 0; --d) div *= (unsigned)g.src[d];
    for (int d = nd - 1; d >= 0; --d) {
        unsigned f = (unsigned)g.fft[d], sr = (unsigned)g.src[d];
        div /= sr;
        index = index * f + (f - (position / div + (unsigned)mn[d]) % sr - 1u);
    }
    return index < (unsigned)g.N ? int(index) : -1;
}

// slot `warp` of a batch (one warp)
__device__ __forceinline__ void prep_sim_warp(const SimPrepArgs &A, const int warp, const int lane) {
    if (warp >= A.nslots) return;
    const int i = A.nodes[warp];
    const unsigned pv = A.path[A.begin + i];
    // -fs: the path entry is a cell value (cell * nvar + variable)
    const unsigned cell = A.full ? pv / unsigned(A.nvar) : pv;
    const int cnt = A.nb_count[i];
    const int nd = A.g.nd;
    const NodeGeom ng = node_geometry(A, i, cell, lane);
    Slot s;
    s.node = i;
    s.cell = cell;
    s.var = A.full ? int(pv % unsigned(A.nvar)) : 0;
    s.seed = A.seeds[i];
    const float lk = ng.lk;
    const int Ki = ng.Ki;
    s.K = Ki;
    s.sel = selected_index(s.seed, lk, A.nti);
    if (s.sel < 0) s.sel = 0;
    if (s.sel > Ki - 1) s.sel = Ki - 1;   // unreachable for k >= 1 and seeds in [0,1)
    s.flags = 0;
    s.nterms = 0;
    s.excl = -1;
    s.cmask_base = 0;
    int mn[QSK_MAXD];
#pragma unroll
    for (int d = 0; d < QSK_MAXD; ++d) {
        mn[d] = ng.mn[d];
        s.mn[d] = ng.mn[d];
        s.lo[d] = ng.lo[d];
    }
    if (ng.skip) {
        s.flags |= SLOT_SKIP;
    } else {
        if (ng.nvalid < Ki) s.flags |= SLOT_EMIT_MASKED;
        // terms: neighbours in order, variables in order; zero-weight / NaN skipped
        int base_out = 0;
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            int j = j0 + lane;
            Term tl[8];
            int nt = 0;
            if (j < cnt) {
                int t = A.nb_tpl[(long long)i * A.n + j];
                unsigned nc = A.nb_cell[(long long)i * A.n + j];
                long long d_flat = 0;
                for (int d = 0; d < nd; ++d) d_flat += (long long)(A.tpl[t * nd + d] - mn[d]) * A.g.sstride[d];
                for (int v = 0; v < A.nvar && v < 4; ++v) {
                    // a variable takes values from its first n_v neighbours only
                    // (simulation.hpp:476-497)
                    if (A.full) {
                        if (!((A.nb_mask[(long long)i * A.n + j] >> v) & 1u)) continue;
                    } else if (A.node_nv && j >= A.node_nv[(long long)i * A.nvar + v]) {
                        continue;
                    }
                    float val = (nc == cell && !A.full) ? A.init[(long long)nc * A.nvar + v]
                                                        : A.state[(long long)nc * A.nvar + v];
                    float w = A.wtab[t * A.nvar + v];
                    if (isnan(val) || w == 0.f) continue;
                    Term tm;
                    tm.base = int((long long)v * A.g.N - d_flat);
                    if (A.types[v] == 0 && A.missing) {
                        // regular output: -w TI^2 + 2wv TI - ((w v) v) mask; overlap: w mask
                        tm.op = OP_SQLINM;
                        tm.a = -w;
                        tm.b = 2.f * __fmul_rn(w, val);
                        tl[nt++] = tm;
                        Term pl;
                        pl.base = tm.base;
                        pl.op = OP_NOP;
                        pl.a = -__fmul_rn(__fmul_rn(w, val), val);
                        pl.b = w;
                        tl[nt++] = pl;
                        continue;
                    }
                    if (A.types[v] == 0) {
                        tm.op = OP_SQLIN;
                        tm.a = -w;
                        tm.b = 2.f * __fmul_rn(w, val);
                    } else {
                        tm.op = OP_EQ;
                        tm.a = w;
                        tm.b = val;
                    }
                    tl[nt++] = tm;
                }
            }
            // order-preserving compaction across the warp
            int incl = nt;
            for (int off = 1; off < 32; off <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += y;
            }
            int excl = incl - nt;
            int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int q = 0; q < nt; ++q) {
                int o = base_out + excl + q;
                if (o < A.maxterms) A.terms[(long long)warp * A.maxterms + o] = tl[q];
            }
            base_out += total;
        }
        if (base_out > A.maxterms) {
            if (lane == 0) atomicExch(A.status, DEV_TOO_MANY_TERMS);
            base_out = A.maxterms;
        }
        s.nterms = base_out;
        if (A.missing) {
            s.flags |= SLOT_MISSING;
            long long fmn = 0;
            for (int d = 0; d < nd; ++d) fmn += (long long)mn[d] * A.g.sstride[d];
            s.cmask_base = int((long long)A.mask_layer * A.g.N + fmn);
        }
        if (A.no_verbatim && cnt > 1 && !A.full) {
            // the TI cell continuing neighbour 1's source is excluded
            const int t1 = A.nb_tpl[(long long)i * A.n + 1];
            const unsigned c1 = A.nb_cell[(long long)i * A.n + 1];
            s.excl = verbatim_excl(A.g, A.tpl + t1 * nd, A.id_image[c1], mn);
        }
    }
    s.vcell = 0;
    s.vtpl = -1;
    if (lane == 0) A.slots[warp] = s;
}

__global__ void k_prep_sim(SimPrepArgs A) {
    griddep_launch();   // a programmatic successor (k_tc_nodes) may begin launching
    prep_sim_warp(A, int((blockIdx.x * blockDim.x + threadIdx.x) >> 5), int(threadIdx.x & 31));
}

// A tensor-core level's exact terms (k_prep_sim) and node rows (k_tc_nodes)
// in one grid: blocks [0, prep_blocks) prepare the slots, the others write
// the rows.  Neither part reads what the other writes (both read only the
// neighbours, values and seeds of earlier levels), so they need no order.
__global__ void k_prep_tc_nodes(SimPrepArgs P, TcNodeArgs T, unsigned prep_blocks) {
    griddep_launch();   // the shortlist (a programmatic successor) may begin launching
    const int lane = int(threadIdx.x & 31);
    if (blockIdx.x < prep_blocks) prep_sim_warp(P, int((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane);
    else tc_nodes_warp(T, int(((blockIdx.x - prep_blocks) * blockDim.x + threadIdx.x) >> 5), lane);
}

// ---------------------------------------------------------------------------
// fused map + record filter
// ---------------------------------------------------------------------------
template <int KF>
__global__ void __launch_bounds__(256) k_map_records(MapArgs A) {
    extern __shared__ Term sterm[];
    __shared__ Slot ss;
    const int b = blockIdx.y;
    if (threadIdx.x == 0) ss = A.slots[b];
    __syncthreads();
    if (ss.flags & SLOT_SKIP) return;
    const int nt = ss.nterms;
    const Term *src = A.terms + (long long)b * A.maxterms;
    for (int t = threadIdx.x; t < nt; t += blockDim.x) sterm[t] = src[t];
    __syncthreads();

    const Geom &g = A.g;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const bool emit_masked = (ss.flags & SLOT_EMIT_MASKED) != 0;
    // a valid scan position used for address-safe dummy gathers; with no valid
    // position at all every entry is masked and no gather is issued
    long long m_safe = 0;
    bool any_valid = true;
    for (int d = 0; d < g.nd; ++d) {
        m_safe += (long long)ss.lo[d] * g.sstride[d];
        any_valid &= ss.lo[d] < g.fft[d];
    }
    const int nt_eff = any_valid ? nt : 0;
    if (!any_valid) m_safe = 0;
    const unsigned usafe = (unsigned)m_safe;
    const unsigned uN = (unsigned)g.N;

    const int seg_begin = blockIdx.x * A.segs_per_cta;
    int seg_end = seg_begin + A.segs_per_cta;
    if (seg_end > g.nseg) seg_end = g.nseg;
    float *rv = A.rec_val + (long long)b * g.nseg * QSK_SEG;
    int *ri = A.rec_idx + (long long)b * g.nseg * QSK_SEG;

    for (int sg = seg_begin + warp; sg < seg_end; sg += nwarps) {
        const unsigned base = (unsigned)sg * QSK_SEG;
        unsigned mm[4];
        bool valid[4], exists[4];
        float acc[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            unsigned m = base + 32 * r + lane;
            exists[r] = m < uN;
            bool ok = exists[r] && any_valid;
            if (ok) {
#pragma unroll
                for (int d = 0; d < QSK_MAXD; ++d)
                    if (d < g.nd) ok &= (int)((m / (unsigned)g.sstride[d]) % (unsigned)g.fft[d]) >= ss.lo[d];
            }
            valid[r] = ok;
            mm[r] = ok ? m : usafe;
            acc[r] = 0.f;
        }
        float crs[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) crs[r] = 0.f;
        for (int t = 0; t < nt_eff; ++t) {
            const Term tm = sterm[t];
            const float *lp = A.layers + tm.base;
            float x[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) x[r] = __ldg(lp + mm[r]);
            if (tm.op == OP_SQLIN) {
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    acc[r] = __fmaf_rn(tm.a, __fmul_rn(x[r], x[r]), acc[r]);
                    acc[r] = __fmaf_rn(tm.b, x[r], acc[r]);
                }
            } else if (tm.op == OP_EQ) {
#pragma unroll
                for (int r = 0; r < 4; ++r) acc[r] = (x[r] == tm.b) ? __fadd_rn(acc[r], tm.a) : acc[r];
            } else if (tm.op == OP_LIN) {
#pragma unroll
                for (int r = 0; r < 4; ++r) acc[r] = __fmaf_rn(tm.a, x[r], acc[r]);
            } else if (tm.op == OP_LINX) {
#pragma unroll
                for (int r = 0; r < 4; ++r) crs[r] = __fmaf_rn(tm.a, x[r], crs[r]);
            } else if (tm.op == OP_SQLINM) {
                const Term pl = sterm[t + 1];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const bool in = !isnan(x[r]);
                    const float x0 = in ? x[r] : 0.f;
                    const float mk = in ? 1.f : 0.f;
                    acc[r] = __fmaf_rn(tm.a, __fmul_rn(x0, x0), acc[r]);
                    acc[r] = __fmaf_rn(tm.b, x0, acc[r]);
                    acc[r] = __fmaf_rn(pl.a, mk, acc[r]);
                    crs[r] = __fmaf_rn(pl.b, mk, crs[r]);
                }
                ++t;
            }
        }
        if (ss.flags & SLOT_MISSING) {
            // overlap masked by the centre, then -|S/c^4| (-inf where c == 0);
            // positions outside the border are NaN in the reference
            // (quantileSamplingModule.hpp:507-516, CPUThreadDevice.cpp:501-524)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const float cm = valid[r] ? __ldg(A.layers + ss.cmask_base + (long long)mm[r]) : 0.f;
                const float c = __fmul_rn(crs[r], cm);
                const float c4 = __fmul_rn(__fmul_rn(__fmul_rn(c, c), c), c);
                float e = -fabsf(__fdiv_rn(acc[r], c4));
                if (c == 0.f) e = -CUDART_INF_F;
                acc[r] = valid[r] ? e : CUDART_NAN_F;
            }
        }
        // verbatim exclusion (one index, or the radius mask): -inf written over
        // the map after the compensation, at masked positions too, where it
        // replaces the NaN border of a missing-data map
        // (quantileSamplingModule.hpp:518-523, CPUThreadDevice.cpp:310-342)
        bool hit[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) hit[r] = exists[r] && (int)(base + 32 * r + lane) == ss.excl;
        if (A.xmask) {
            const unsigned *xm = A.xmask + (long long)b * A.xwords;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const unsigned m = base + 32 * r + lane;
                if (exists[r] && ((xm[m >> 5] >> (m & 31)) & 1u)) hit[r] = true;
            }
        }
        // a masked position is an explicit record when the slot emits masked
        // entries, or when it is an excluded one of a missing-data map (-inf
        // instead of NaN); otherwise the replay counts it as an implicit -inf
        const bool missing = (ss.flags & SLOT_MISSING) != 0;
        // warp prefix top-KF over the segment in scan order; records are the
        // positions not below the K-th best of everything before them in the
        // segment (a superset of the global triggers).
        float carry[KF];
#pragma unroll
        for (int q = 0; q < KF; ++q) carry[q] = -CUDART_INF_F;
        int count = 0;
        float segmax = -CUDART_INF_F;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float xval = hit[r] ? -CUDART_INF_F : valid[r] ? acc[r] : (missing ? CUDART_NAN_F : -CUDART_INF_F);
            segmax = fmaxf(segmax, xval);
            // a NaN score never compares true in the reservoir (fKb.hpp), so it
            // is never a record and must not raise the prefix K-th best: it
            // enters the scan as -inf (fminf/fmaxf would turn it into +inf)
            float st[KF];
            st[0] = isnan(xval) ? -CUDART_INF_F : xval;
#pragma unroll
            for (int q = 1; q < KF; ++q) st[q] = -CUDART_INF_F;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                float rcv[KF], mrg[KF];
#pragma unroll
                for (int q = 0; q < KF; ++q) rcv[q] = __shfl_up_sync(0xffffffffu, st[q], off);
                if (lane >= off) {
                    topk_merge<KF>(st, rcv, mrg);
#pragma unroll
                    for (int q = 0; q < KF; ++q) st[q] = mrg[q];
                }
            }
            float ex[KF], pre[KF];
#pragma unroll
            for (int q = 0; q < KF; ++q) {
                float y = __shfl_up_sync(0xffffffffu, st[q], 1);
                ex[q] = lane == 0 ? -CUDART_INF_F : y;
            }
            topk_merge<KF>(carry, ex, pre);
            const float kth = pre[KF - 1];
            const bool rec = exists[r] && (xval >= kth) && (valid[r] || emit_masked || (hit[r] && missing));
            const unsigned bal = __ballot_sync(0xffffffffu, rec);
            if (rec) {
                const int o = count + __popc(bal & lanemask_lt());
                rv[base + o] = xval;
                ri[base + o] = int(base + 32 * r + lane);
            }
            count += __popc(bal);
            float last[KF], nc[KF];
#pragma unroll
            for (int q = 0; q < KF; ++q) last[q] = __shfl_sync(0xffffffffu, st[q], 31);
            topk_merge<KF>(carry, last, nc);
#pragma unroll
            for (int q = 0; q < KF; ++q) carry[q] = nc[q];
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) segmax = fmaxf(segmax, __shfl_xor_sync(0xffffffffu, segmax, off));
        if (lane == 0) {
            A.rec_cnt[(long long)b * g.nseg + sg] = count;
            A.rec_max[(long long)b * g.nseg + sg] = segmax;
        }
    }
}

// ---------------------------------------------------------------------------
// mt19937 (published algorithm: Matsumoto & Nishimura 1998) with the
// conversion of std::uniform_real_distribution<float>(0,1) in libstdc++
// (generate_canonical<float,24>: float(u32) * 2^-32, values >= 1 clamped to
// the largest float below 1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned mt_temper(unsigned y) {
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

__device__ __forceinline__ float mt_unit(unsigned y) {
    float u = __fmul_rn(__uint2float_rn(y), 2.3283064365386963e-10f);
    return u >= 1.f ? 0x1.fffffep-1f : u;
}

__device__ __forceinline__ unsigned mt_mix(unsigned a, unsigned b, unsigned c) {
    unsigned y = (a & 0x80000000u) | (b & 0x7fffffffu);
    return c ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
}

// warp-cooperative regeneration of the 624-word state (3 dependency phases);
// with OUT, draw k of the new block (tempered, converted) goes to out[k].
// Branch-free: lanes past the end of a phase compute a clamped element and
// store it into their own dummy slots (mt[624 + lane], dummy[lane]), which
// keeps the phases free of divergent stores (3x faster than predicated ones).
template <bool OUT>
__device__ __forceinline__ void mt_twist(unsigned *mt, int lane, float *out, float *dummy) {
    unsigned nv[8];
    int kk[8];
    // phase A: k in [0,227): old x[k], x[k+1], x[k+397]
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = lane + 32 * q;
        const int kc = k < 227 ? k : 226;
        kk[q] = k < 227 ? k : -1;
        nv[q] = mt_mix(mt[kc], mt[kc + 1], mt[kc + 397]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = kk[q];
        mt[k >= 0 ? k : 624 + lane] = nv[q];
        if (OUT) *(k >= 0 ? out + k : dummy + lane) = mt_unit(mt_temper(nv[q]));
    }
    __syncwarp();
    // phase B: k in [227,454): old x[k], x[k+1]; new x[k-227]
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = 227 + lane + 32 * q;
        const int kc = k < 454 ? k : 453;
        kk[q] = k < 454 ? k : -1;
        nv[q] = mt_mix(mt[kc], mt[kc + 1], mt[kc - 227]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int k = kk[q];
        mt[k >= 0 ? k : 624 + lane] = nv[q];
        if (OUT) *(k >= 0 ? out + k : dummy + lane) = mt_unit(mt_temper(nv[q]));
    }
    __syncwarp();
    // phase C: k in [454,623): old x[k], x[k+1]; new x[k-227]
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int k = 454 + lane + 32 * q;
        const int kc = k < 623 ? k : 622;
        kk[q] = k < 623 ? k : -1;
        nv[q] = mt_mix(mt[kc], mt[kc + 1], mt[kc - 227]);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        const int k = kk[q];
        mt[k >= 0 ? k : 624 + lane] = nv[q];
        if (OUT) *(k >= 0 ? out + k : dummy + lane) = mt_unit(mt_temper(nv[q]));
    }
    __syncwarp();
    // k = 623: old x[623], new x[0], new x[396]
    const unsigned y = mt_mix(mt[623], mt[0], mt[396]);
    __syncwarp();
    if (lane == 0) {
        mt[623] = y;
        if (OUT) out[623] = mt_unit(mt_temper(y));
    }
    __syncwarp();
}

// generator.seed(seedFromUnitFloat(seed) + 0)  (quantileSamplingModule.hpp:45-49,533-534):
// the standard mt19937 initialisation, serial, on the calling thread
__device__ __forceinline__ void mt_seed(unsigned *mt, float sd) {
    unsigned x;
    if (!isfinite(sd) || sd <= 0.f) x = 0u;
    else if (sd >= 1.f) x = 0xffffffffu;
    else x = (unsigned)floor((double)sd * 4294967295.0);
    mt[0] = x;
    for (int i = 1; i < 624; ++i) {
        x = 1812433253u * (x ^ (x >> 30)) + (unsigned)i;
        mt[i] = x;
    }
}

// ---------------------------------------------------------------------------
// replay of the k-biggest scan + draw + write-back; one warp per slot
// ---------------------------------------------------------------------------
#define RP_WARPS 4
#define REC_CAP 1024          // records (padded to 4 per segment) of one tie super-run
#define TAB_CAP 128           // segments of one tie super-run
#define RNG_BUF (2 * REC_CAP + 640)   // draws of one super-run + one block
#define SEG_WIN 256           // record counts and maxima of SEG_WIN segments staged per warp
#define TEAM_MAX 8            // warps of one slot's team

struct __align__(16) WarpShared {
    float rv_s[REC_CAP];      // super-run records (values), 16-byte aligned for cp.async
    int ri_s[REC_CAP];        // and their scan indices
    unsigned mt[624 + 32];    // + one dummy word per lane (branch-free twist)
    float buf[RNG_BUF];
    float dummy[32];
    int tseg[TAB_CAP];        // super-run segments, their first padded record, record count
    int tpre[TAB_CAP];
    int tcnt[TAB_CAP];
    int wc[SEG_WIN];          // record counts and maxima of segments [wbase, wbase + SEG_WIN)
    float wm[SEG_WIN];
    // a team of warps on one slot (k_replay with W > 1): the command warp 0
    // posts, and the per-warp tie counts and slot maps of a super-run
    int cmd, cmd_off, cmd_tp, cmd_xes, cmd_k, cmd_rp;
    unsigned cmd_cpt;
    float cmd_v;
    int tw_sum[TEAM_MAX];
    int tw_map[TEAM_MAX][QSK_KMAX];
};

enum TeamCommand : int { CMD_EXIT = 0, CMD_TWIST = 1, CMD_TWIST_OUT = 2, CMD_SUPER = 3 };

// barrier 1 over the team's threads (barrier 0 stays free for __syncthreads)
__device__ __forceinline__ void team_bar(int nthreads) { asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory"); }

// mt_twist with the elements of each dependency phase spread over the NT
// (>= 128) threads of a team
template <bool OUT>
__device__ void mt_twist_team(unsigned *mt, int tid, int NT, float *out) {
    unsigned nv[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int k = tid + i * NT;
        nv[i] = k < 227 ? mt_mix(mt[k], mt[k + 1], mt[k + 397]) : 0u;
    }
    team_bar(NT);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int k = tid + i * NT;
        if (k < 227) {
            mt[k] = nv[i];
            if (OUT) out[k] = mt_unit(mt_temper(nv[i]));
        }
    }
    team_bar(NT);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int k = 227 + tid + i * NT;
        nv[i] = k < 454 ? mt_mix(mt[k], mt[k + 1], mt[k - 227]) : 0u;
    }
    team_bar(NT);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int k = 227 + tid + i * NT;
        if (k < 454) {
            mt[k] = nv[i];
            if (OUT) out[k] = mt_unit(mt_temper(nv[i]));
        }
    }
    team_bar(NT);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int k = 454 + tid + i * NT;
        nv[i] = k < 623 ? mt_mix(mt[k], mt[k + 1], mt[k - 227]) : 0u;
    }
    team_bar(NT);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int k = 454 + tid + i * NT;
        if (k < 623) {
            mt[k] = nv[i];
            if (OUT) out[k] = mt_unit(mt_temper(nv[i]));
        }
    }
    team_bar(NT);
    if (tid == 0) {
        const unsigned y = mt_mix(mt[623], mt[0], mt[396]);
        mt[623] = y;
        if (OUT) out[623] = mt_unit(mt_temper(y));
    }
    team_bar(NT);
}

// Make segments [q0, q0 + 32) readable from the window (w.wc / w.wm at q - wbase).
// The scan only moves forward, so a miss restages the window from q0 on.
__device__ __forceinline__ void win_cover(WarpShared &w, int &wbase, int q0, int nseg, const int *rc, const float *rm,
                                          int lane) {
    if (q0 >= wbase && q0 + 32 <= wbase + SEG_WIN) return;
    __syncwarp();
    wbase = q0;
    int c[SEG_WIN / 32];
    float m[SEG_WIN / 32];
#pragma unroll
    for (int i = 0; i < SEG_WIN / 32; ++i) {
        const int q = q0 + lane + 32 * i;
        c[i] = q < nseg ? rc[q] : 0;
        m[i] = q < nseg ? rm[q] : -CUDART_INF_F;
    }
#pragma unroll
    for (int i = 0; i < SEG_WIN / 32; ++i) {
        w.wc[lane + 32 * i] = c[i];
        w.wm[lane + 32 * i] = m[i];
    }
    __syncwarp();
}

// One MT19937 block of the slot's stream: regenerated by warp 0 alone (W ==
// 1), or by the whole team, which warp 0 wakes with a command (W > 1).
template <int W, bool OUT>
__device__ __forceinline__ void rng_block(WarpShared &w, int lane, float *out) {
    if constexpr (W == 1) {
        mt_twist<OUT>(w.mt, lane, out, w.dummy);
    } else {
        __syncwarp();
        if (lane == 0) {
            w.cmd = OUT ? CMD_TWIST_OUT : CMD_TWIST;
            w.cmd_off = OUT ? int(out - w.buf) : 0;
        }
        team_bar(32 * W);
        mt_twist_team<OUT>(w.mt, threadIdx.x, 32 * W, out);
    }
}

// Draw buffer with warp-replicated read pointer: rp/len live in registers of
// every lane (all lanes execute the same control flow).
template <int W>
__device__ __forceinline__ void rng_refill(WarpShared &w, int lane, int &rp, int &len) {
    const int unread = len - rp;   // <= 2 * REC_CAP by construction
    // move the unread draws to the front (destinations never overtake sources)
    __syncwarp();
    for (int q = 0; 32 * q < unread; ++q) {
        const int i = lane + 32 * q;
        const float v = i < unread ? w.buf[rp + i] : 0.f;
        __syncwarp();
        if (i < unread) w.buf[i] = v;
        __syncwarp();
    }
    rng_block<W, true>(w, lane, w.buf + unread);
    len = unread + 624;
    rp = 0;
}

template <int W>
__device__ __forceinline__ void rng_ensure(WarpShared &w, int lane, int &rp, int &len, int need) {
    if (len - rp < need) rng_refill<W>(w, lane, rp, len);
}

// at least `need` (<= 2 * REC_CAP) unread draws in the buffer
template <int W>
__device__ void rng_ensure_many(WarpShared &w, int lane, int &rp, int &len, int need) {
    if (len - rp >= need) return;
    const int unread = len - rp;
    __syncwarp();
    for (int q = 0; 32 * q < unread; ++q) {
        const int i = lane + 32 * q;
        const float v = i < unread ? w.buf[rp + i] : 0.f;
        __syncwarp();
        if (i < unread) w.buf[i] = v;
        __syncwarp();
    }
    len = unread;
    rp = 0;
    while (len < need) {
        rng_block<W, true>(w, lane, w.buf + len);
        len += 624;
    }
}

// advance the stream by n draws; whole blocks of 624 only regenerate the state
template <int W>
__device__ void rng_skip(WarpShared &w, int lane, int &rp, int &len, long long n) {
    const long long avail = len - rp;
    if (n <= avail) {
        rp += int(n);
        return;
    }
    n -= avail;
    rp = len;
    while (n > 624) {
        rng_block<W, false>(w, lane, nullptr);
        n -= 624;
    }
    rng_refill<W>(w, lane, rp, len);
    rp += int(n);
}

template <int KM>
__device__ __forceinline__ float sel_f(const float (&a)[KM], int i) {
    float r = a[0];
#pragma unroll
    for (int s = 1; s < KM; ++s) r = (s == i) ? a[s] : r;
    return r;
}
template <int KM>
__device__ __forceinline__ int sel_i(const int (&a)[KM], int i) {
    int r = a[0];
#pragma unroll
    for (int s = 1; s < KM; ++s) r = (s == i) ? a[s] : r;
    return r;
}
template <int KM>
__device__ __forceinline__ unsigned sel_u(const unsigned (&a)[KM], int i) {
    unsigned r = a[0];
#pragma unroll
    for (int s = 1; s < KM; ++s) r = (s == i) ? a[s] : r;
    return r;
}

// One step of the reference's k-biggest scan for up to 32 consecutive
// candidates at once (one per lane, lanes in scan order).  The value state is
// a prefix top-K (associative merge), the tie counter cpt a composition of
// "add" / "reset" functions, the draws a prefix count, and the position
// updates of each trigger (swap of the tail slot, insertion, reservoir
// replacement) slot maps whose composition is reduced across the warp.
// State (cv, cp, cpt, rp) is replicated in all lanes.
template <int KM>
__device__ __forceinline__ void replay_chunk(int K, bool valid, float v, int m, float (&cv)[KM], unsigned (&cp)[KM],
                                             unsigned &cpt, int &rp, const float *buf, int lane) {
    const unsigned FULL = 0xffffffffu;
    // 1. exclusive prefix top-K of the chunk's values, merged with the state
    float st[KM];
    st[0] = valid ? v : -CUDART_INF_F;
#pragma unroll
    for (int s = 1; s < KM; ++s) st[s] = -CUDART_INF_F;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        float rcv[KM], mrg[KM];
#pragma unroll
        for (int s = 0; s < KM; ++s) rcv[s] = __shfl_up_sync(FULL, st[s], off);
        if (lane >= off) {
            topk_merge<KM>(st, rcv, mrg);
#pragma unroll
            for (int s = 0; s < KM; ++s) st[s] = mrg[s];
        }
    }
    float ex[KM], pre[KM];
#pragma unroll
    for (int s = 0; s < KM; ++s) {
        float y = __shfl_up_sync(FULL, st[s], 1);
        ex[s] = lane == 0 ? -CUDART_INF_F : y;
    }
    topk_merge<KM>(cv, ex, pre);
    const float kth = sel_f<KM>(pre, K - 1);
    const bool trig = valid && (v >= kth);
    const bool gt = trig && (v > kth);
    int xes = 0, q = 0;
#pragma unroll
    for (int s = 0; s < KM; ++s) {
        if (s < K && pre[s] == kth) xes++;
        if (s < K - 1 && pre[s] >= v) q++;
    }
    // 2. cpt as functions c -> r ? a : c + a, exclusive scan in lane order
    int fr = 0, fa = 0;
    if (trig) {
        if (gt && xes == 1) { fr = 1; fa = 0; }
        else { fr = 0; fa = 1; }
    }
    int er = 0, ea = 0;   // exclusive composite
    {
        int ir = fr, ia = fa;   // inclusive composite (scan)
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int rr = __shfl_up_sync(FULL, ir, off), ra = __shfl_up_sync(FULL, ia, off);
            if (lane >= off) {
                // earlier (rr,ra) then later (ir,ia)
                if (!ir) { ir = rr; ia = ra + ia; }
            }
        }
        int pr = __shfl_up_sync(FULL, ir, 1), pa = __shfl_up_sync(FULL, ia, 1);
        if (lane > 0) { er = pr; ea = pa; }
        // total composite from lane 31 for the state update below
        int tr = __shfl_sync(FULL, ir, 31), ta = __shfl_sync(FULL, ia, 31);
        const unsigned before = er ? unsigned(ea) : cpt + unsigned(ea);
        const unsigned after = fr ? 0u : before + unsigned(fa);
        // 3. draw offsets: 1 draw per trigger, a second one per tie
        const unsigned b1 = __ballot_sync(FULL, trig), b2 = __ballot_sync(FULL, trig && !gt);
        const unsigned lt = lanemask_lt();
        const int off = __popc(b1 & lt) + __popc(b2 & lt);
        int o[KM];
#pragma unroll
        for (int s = 0; s < KM; ++s) o[s] = s;
        if (trig) {
            const float u1 = buf[rp + off];
            int x = K - xes + int(floorf(__fmul_rn(u1, (float)xes)));
            if (x > K - 1) x = K - 1;
            bool write = false;
            if (!gt) {
                const float u2 = buf[rp + off + 1];
                write = __fmul_rn(__uint2float_rn(unsigned(xes) + after), u2) < (float)xes;
            }
            int sig[KM];
#pragma unroll
            for (int s = 0; s < KM; ++s) sig[s] = (s == x) ? K - 1 : ((s == K - 1) ? x : s);
            if (gt) {
#pragma unroll
                for (int s = 0; s < KM; ++s) {
                    if (s < K) {
                        int prevs = s > 0 ? sig[s > 0 ? s - 1 : 0] : 0;
                        o[s] = s < q ? sig[s] : (s == q ? -(m + 1) : prevs);
                    }
                }
            } else {
#pragma unroll
                for (int s = 0; s < KM; ++s)
                    if (s < K) o[s] = (write && s == K - 1) ? -(m + 1) : sig[s];
            }
        }
        // 4. compose the slot maps in lane order (tree reduction to lane 0)
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            int later[KM];
#pragma unroll
            for (int s = 0; s < KM; ++s) later[s] = __shfl_down_sync(FULL, o[s], d);
            if ((lane & (2 * d - 1)) == 0 && lane + d < 32) {
                int c[KM];
#pragma unroll
                for (int s = 0; s < KM; ++s) c[s] = later[s] < 0 ? later[s] : sel_i<KM>(o, later[s]);
#pragma unroll
                for (int s = 0; s < KM; ++s) o[s] = c[s];
            }
        }
        unsigned np[KM];
#pragma unroll
        for (int s = 0; s < KM; ++s) {
            int t = __shfl_sync(FULL, o[s], 0);
            np[s] = t < 0 ? unsigned(-(t + 1)) : sel_u<KM>(cp, t);
        }
#pragma unroll
        for (int s = 0; s < KM; ++s) cp[s] = np[s];
        // 5. state values, cpt, draw pointer
        float last[KM], nv[KM];
#pragma unroll
        for (int s = 0; s < KM; ++s) last[s] = __shfl_sync(FULL, st[s], 31);
        topk_merge<KM>(cv, last, nv);
#pragma unroll
        for (int s = 0; s < KM; ++s) cv[s] = nv[s];
        cpt = tr ? unsigned(ta) : cpt + unsigned(ta);
        rp += __popc(b1) + __popc(b2);
    }
}

// Steady-state fast path: every value of the state equals the K-th (so
// xes = K and a trigger can only tie) and no candidate of the chunk exceeds
// it.  Each tie uses two draws and increments cpt; lane ranks give both.
template <int KM>
__device__ __forceinline__ void replay_chunk_ties(int K, bool tie, int m, unsigned (&cp)[KM], unsigned &cpt, int &rp,
                                                  const float *buf, int lane) {
    const unsigned FULL = 0xffffffffu;
    const unsigned bt = __ballot_sync(FULL, tie);
    const int rank = __popc(bt & lanemask_lt());
    int o[KM];
#pragma unroll
    for (int s = 0; s < KM; ++s) o[s] = s;
    if (tie) {
        const float u1 = buf[rp + 2 * rank];
        const float u2 = buf[rp + 2 * rank + 1];
        int x = int(floorf(__fmul_rn(u1, (float)K)));
        if (x > K - 1) x = K - 1;
        const unsigned after = cpt + unsigned(rank) + 1u;
        const bool write = __fmul_rn(__uint2float_rn(unsigned(K) + after), u2) < (float)K;
#pragma unroll
        for (int s = 0; s < KM; ++s) {
            if (s < K) {
                int sig = (s == x) ? K - 1 : ((s == K - 1) ? x : s);
                o[s] = (write && s == K - 1) ? -(m + 1) : sig;
            }
        }
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int later[KM];
#pragma unroll
        for (int s = 0; s < KM; ++s) later[s] = __shfl_down_sync(FULL, o[s], d);
        if ((lane & (2 * d - 1)) == 0) {
            int c[KM];
#pragma unroll
            for (int s = 0; s < KM; ++s) c[s] = later[s] < 0 ? later[s] : sel_i<KM>(o, later[s]);
#pragma unroll
            for (int s = 0; s < KM; ++s) o[s] = c[s];
        }
    }
    unsigned np[KM];
#pragma unroll
    for (int s = 0; s < KM; ++s) {
        int t = __shfl_sync(FULL, o[s], 0);
        np[s] = t < 0 ? unsigned(-(t + 1)) : sel_u<KM>(cp, t);
    }
#pragma unroll
    for (int s = 0; s < KM; ++s) cp[s] = np[s];
    const int nt = __popc(bt);
    cpt += unsigned(nt);
    rp += 2 * nt;
}

// A few candidates (the lanes of cand, in scan order): the reference's scan
// step (fKb.hpp) applied to one trigger after the other, warp-uniformly.
// A trigger v >= K-th draws x among the xes tail slots holding the K-th and
// swaps it with slot K-1; above the K-th it is inserted after the values
// >= v (the last slot drops out, cpt restarts at 0 when the K-th was unique
// and counts on otherwise); equal to the K-th it replaces slot K-1 with
// probability xes / (xes + cpt + 1) (a second draw) and cpt counts on.
template <int KM>
__device__ __forceinline__ void replay_scalar(int K, unsigned cand, float v, int m, float (&cv)[KM],
                                              unsigned (&cp)[KM], unsigned &cpt, int &rp, const float *buf) {
    const unsigned FULL = 0xffffffffu;
    while (cand) {
        const int l = __ffs(cand) - 1;
        cand &= cand - 1u;
        const float xv = __shfl_sync(FULL, v, l);
        const unsigned xm = (unsigned)__shfl_sync(FULL, m, l);
        const float kth = sel_f<KM>(cv, K - 1);
        if (!(xv >= kth)) continue;
        const bool gt = xv > kth;
        int xes = 0, q = 0;
#pragma unroll
        for (int s = 0; s < KM; ++s) {
            if (s < K && cv[s] == kth) xes++;
            if (s < K - 1 && cv[s] >= xv) q++;
        }
        int x = K - xes + int(floorf(__fmul_rn(buf[rp], (float)xes)));
        if (x > K - 1) x = K - 1;
        const unsigned px = sel_u<KM>(cp, x), pk = sel_u<KM>(cp, K - 1);
        unsigned sw[KM];
#pragma unroll
        for (int s = 0; s < KM; ++s) sw[s] = (s == x) ? pk : ((s == K - 1) ? px : cp[s]);
        if (gt) {
#pragma unroll
            for (int s = 0; s < KM; ++s)
                if (s < K) cp[s] = s < q ? sw[s] : (s == q ? xm : sw[s > 0 ? s - 1 : 0]);
            topk_insert<KM>(cv, xv);
            cpt = (xes == 1) ? 0u : cpt + 1u;
            rp += 1;
        } else {
            const unsigned after = cpt + 1u;
            const bool write = __fmul_rn(__uint2float_rn(unsigned(xes) + after), buf[rp + 1]) < (float)xes;
#pragma unroll
            for (int s = 0; s < KM; ++s) cp[s] = (write && s == K - 1) ? xm : sw[s];
            cpt = after;
            rp += 2;
        }
    }
}

__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One tie super-run: no record of the run exceeds the K-th value V of the
// state, so the state's values stay as they are, every record equal to V is a
// tie (two draws, cpt + 1, a swap inside the xes tail slots that hold V and a
// possible replacement at K-1) and the others are no-ops.  The run's segments
// (w.tseg/tpre/tcnt, E entries, Tp padded records) arrive in shared memory by
// the 16-byte asynchronous copies issued while they were gathered; lane l
// then owns a contiguous range of the run, counts its ties, composes the slot
// maps of its ties on its own, and one warp reduction combines the 32 lane
// maps in order.
// A super-run on a team of W warps (W > 1): thread t of the team owns
// records [t*P, t*P + P) of the staged run (the parameters warp 0 posted),
// the team's tie counts are scanned through shared memory, every thread
// composes the slot maps of its ties, and the warp maps are composed in warp
// order.  Returns the tie count and the composed map (in every thread).
template <int KM, int W>
__device__ void super_team(WarpShared &w, int tid, int &total, int (&o)[KM]) {
    const unsigned FULL = 0xffffffffu;
    constexpr int NT = 32 * W;
    const int lane = tid & 31, wid = tid >> 5;
    const int Tp = w.cmd_tp, xes = w.cmd_xes, K = w.cmd_k, rp = w.cmd_rp;
    const unsigned cpt = w.cmd_cpt;
    const float V = w.cmd_v;
    // P odd keeps a warp's reads on distinct banks; P <= REC_CAP / NT + 1 bits
    const int P = ((Tp + NT - 1) / NT) | 1;
    const int j0 = min(Tp, tid * P);
    const int j1 = min(Tp, j0 + P);
    unsigned tm = 0u;
    for (int j = j0; j < j1; ++j) tm |= unsigned(w.rv_s[j] == V) << (j - j0);
    const int mine = __popc(tm);
    int incl = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, off);
        if (lane >= off) incl += y;
    }
    if (lane == 31) w.tw_sum[wid] = incl;
    team_bar(NT);
    int before = 0;
    total = 0;
#pragma unroll
    for (int q = 0; q < W; ++q) {
        const int t = w.tw_sum[q];
        before += q < wid ? t : 0;
        total += t;
    }
    int rank = before + incl - mine;
#pragma unroll
    for (int s2 = 0; s2 < KM; ++s2) o[s2] = s2;
    while (tm) {
        const int j = j0 + __ffs(tm) - 1;
        tm &= tm - 1u;
        const float u1 = w.buf[rp + 2 * rank];
        const float u2 = w.buf[rp + 2 * rank + 1];
        int x = K - xes + int(floorf(__fmul_rn(u1, (float)xes)));
        if (x > K - 1) x = K - 1;
        const unsigned after = cpt + unsigned(rank) + 1u;
        const bool write = __fmul_rn(__uint2float_rn(unsigned(xes) + after), u2) < (float)xes;
        const int ox = sel_i<KM>(o, x), ok1 = sel_i<KM>(o, K - 1);
        const int wr = -(w.ri_s[j] + 1);
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) {
            if (s2 == x) o[s2] = ok1;
            if (s2 == K - 1) o[s2] = write ? wr : ox;
        }
        ++rank;
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int later[KM];
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) later[s2] = __shfl_down_sync(FULL, o[s2], d);
        if ((lane & (2 * d - 1)) == 0) {
            int c[KM];
#pragma unroll
            for (int s2 = 0; s2 < KM; ++s2) c[s2] = later[s2] < 0 ? later[s2] : sel_i<KM>(o, later[s2]);
#pragma unroll
            for (int s2 = 0; s2 < KM; ++s2) o[s2] = c[s2];
        }
    }
    if (lane == 0) {
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) w.tw_map[wid][s2] = o[s2];
    }
    team_bar(NT);
#pragma unroll
    for (int s2 = 0; s2 < KM; ++s2) o[s2] = w.tw_map[0][s2];
#pragma unroll
    for (int q = 1; q < W; ++q) {
        int c[KM];
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) {
            const int later = w.tw_map[q][s2];
            c[s2] = later < 0 ? later : sel_i<KM>(o, later);
        }
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) o[s2] = c[s2];
    }
}

// warps 1..W-1 of a team: run the commands warp 0 posts until it is done
template <int KM, int W>
__device__ void team_helper(WarpShared &w) {
    for (;;) {
        team_bar(32 * W);
        const int c = w.cmd;
        if (c == CMD_EXIT) return;
        if (c == CMD_TWIST_OUT) {
            mt_twist_team<true>(w.mt, threadIdx.x, 32 * W, w.buf + w.cmd_off);
        } else if (c == CMD_TWIST) {
            mt_twist_team<false>(w.mt, threadIdx.x, 32 * W, nullptr);
        } else {
            int tot, o[KM];
            super_team<KM, W>(w, threadIdx.x, tot, o);
        }
    }
}

template <int KM, int W>
__device__ void replay_super_run(int K, float V, int xes, int E, int Tp, const float *rv, const int *ri, unsigned (&cp)[KM],
                                 unsigned &cpt, int &rp, int &len, WarpShared &w, int lane) {
    const unsigned FULL = 0xffffffffu;
    cp_async_wait_all();   // the copies issued while the run was gathered
    __syncwarp();
    for (int e = lane; e < E; e += 32) {
        const int c = w.tcnt[e], pre = w.tpre[e];
        for (int k = c; k < ((c + 3) & ~3); ++k) w.rv_s[pre + k] = -CUDART_INF_F;
    }
    __syncwarp();
    if constexpr (W > 1) {
        // draws for every record (at most two per tie), then the team
        rng_ensure_many<W>(w, lane, rp, len, 2 * Tp);
        __syncwarp();
        if (lane == 0) {
            w.cmd = CMD_SUPER;
            w.cmd_tp = Tp;
            w.cmd_v = V;
            w.cmd_xes = xes;
            w.cmd_k = K;
            w.cmd_rp = rp;
            w.cmd_cpt = cpt;
        }
        team_bar(32 * W);
        int total, o[KM];
        super_team<KM, W>(w, threadIdx.x, total, o);
        unsigned np[KM];
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) np[s2] = o[s2] < 0 ? unsigned(-(o[s2] + 1)) : sel_u<KM>(cp, o[s2]);
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) cp[s2] = np[s2];
        cpt += unsigned(total);
        rp += 2 * total;
        __syncwarp();
        return;
    }
    // lane l owns records [l*P, l*P + P); P odd keeps the lanes' reads on
    // distinct shared-memory banks (P <= 33 fits a 64-bit tie mask)
    const int P = ((Tp + 31) >> 5) | 1;
    const int j0 = min(Tp, lane * P);
    const int j1 = min(Tp, j0 + P);
    unsigned long long tmask = 0ull;
#pragma unroll 4
    for (int j = j0; j < j1; ++j) tmask |= (unsigned long long)(w.rv_s[j] == V) << (j - j0);
    const int mine = __popcll(tmask);
    int incl = mine;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(FULL, incl, off);
        if (lane >= off) incl += y;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    int rank = incl - mine;
    rng_ensure_many<W>(w, lane, rp, len, 2 * total);
    int o[KM];
#pragma unroll
    for (int s2 = 0; s2 < KM; ++s2) o[s2] = s2;
    while (tmask) {
        const int j = j0 + __ffsll((long long)tmask) - 1;
        tmask &= tmask - 1ull;
        const float u1 = w.buf[rp + 2 * rank];
        const float u2 = w.buf[rp + 2 * rank + 1];
        int x = K - xes + int(floorf(__fmul_rn(u1, (float)xes)));
        if (x > K - 1) x = K - 1;
        const unsigned after = cpt + unsigned(rank) + 1u;
        const bool write = __fmul_rn(__uint2float_rn(unsigned(xes) + after), u2) < (float)xes;
        // op = (write at K-1) o (swap x, K-1); composed after the lane's earlier ops
        const int ox = sel_i<KM>(o, x), ok1 = sel_i<KM>(o, K - 1);
        const int wr = -(w.ri_s[j] + 1);
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) {
            if (s2 == x) o[s2] = ok1;
            if (s2 == K - 1) o[s2] = write ? wr : ox;
        }
        ++rank;
    }
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int later[KM];
#pragma unroll
        for (int s2 = 0; s2 < KM; ++s2) later[s2] = __shfl_down_sync(FULL, o[s2], d);
        if ((lane & (2 * d - 1)) == 0) {
            int c[KM];
#pragma unroll
            for (int s2 = 0; s2 < KM; ++s2) c[s2] = later[s2] < 0 ? later[s2] : sel_i<KM>(o, later[s2]);
#pragma unroll
            for (int s2 = 0; s2 < KM; ++s2) o[s2] = c[s2];
        }
    }
    unsigned np[KM];
#pragma unroll
    for (int s2 = 0; s2 < KM; ++s2) {
        int t = __shfl_sync(FULL, o[s2], 0);
        np[s2] = t < 0 ? unsigned(-(t + 1)) : sel_u<KM>(cp, t);
    }
#pragma unroll
    for (int s2 = 0; s2 < KM; ++s2) cp[s2] = np[s2];
    cpt += unsigned(total);
    rp += 2 * total;
    __syncwarp();
}

// Tie stream (the state holds K finite values, the K-th is V, xes of them
// equal V): segments from `sg` on whose maximum is V are ties or no-ops,
// those below V are skipped, and the first segment above V ends the stream.  Segments are gathered into super-runs of
// at most REC_CAP padded records and TAB_CAP segments.  Returns the first
// segment above V, or nseg.
template <int KM, int W>
__device__ int replay_tie_stream(int K, float V, int xes, int sg, int nseg, const float *rv, const int *ri, const int *rc,
                                 const float *rm, int &wbase, unsigned (&cp)[KM], unsigned &cpt, int &rp, int &len,
                                 WarpShared &w, int lane) {
    const unsigned FULL = 0xffffffffu;
    const unsigned lt = lanemask_lt();
    for (;;) {
        int E = 0, Tp = 0, stop = -1;
        for (;;) {
            if (sg >= nseg) {
                stop = nseg;
                break;
            }
            win_cover(w, wbase, sg, nseg, rc, rm, lane);
            const int q = sg + lane;
            const int c = w.wc[q - wbase];
            const float m = w.wm[q - wbase];
            const unsigned brk = __ballot_sync(FULL, c > 0 && m > V);
            const unsigned lim = brk ? ((1u << (__ffs(brk) - 1)) - 1u) : FULL;
            const bool elig = ((lim >> lane) & 1u) && c > 0 && m == V;
            const int pc = elig ? ((c + 3) & ~3) : 0;
            int incl = pc;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(FULL, incl, off);
                if (lane >= off) incl += y;
            }
            const unsigned EL = __ballot_sync(FULL, elig);
            const int epos = E + __popc(EL & lt);
            // the limits are monotone in lane order: the taken lanes are a prefix of EL
            const bool take = elig && Tp + incl <= REC_CAP && epos < TAB_CAP;
            const unsigned TK = __ballot_sync(FULL, take);
            if (take) {
                // the segment's records go to the run's buffers right away, so
                // the copies overlap the rest of the gathering
                const int dst = Tp + incl - pc;
                w.tseg[epos] = q;
                w.tpre[epos] = dst;
                w.tcnt[epos] = c;
                const long long src = (long long)q * QSK_SEG;
                for (int k = 0; k < pc; k += 4) {
                    cp_async16(&w.rv_s[dst + k], rv + src + k);
                    cp_async16(&w.ri_s[dst + k], ri + src + k);
                }
            }
            const int hi = TK ? 31 - __clz(TK) : 0;
            const int add = __shfl_sync(FULL, incl, hi);
            if (TK) {
                Tp += add;
                E += __popc(TK);
            }
            const unsigned left = EL & ~TK;
            if (left) {   // capacity reached: the next run starts at the first segment left out
                sg += __ffs(left) - 1;
                break;
            }
            if (brk) {
                sg += __ffs(brk) - 1;
                stop = sg;
                break;
            }
            sg += 32;
        }
        __syncwarp();
        if (E > 0) replay_super_run<KM, W>(K, V, xes, E, Tp, rv, ri, cp, cpt, rp, len, w, lane);
        if (stop >= 0) return stop;
    }
}

// W == 1: RP_WARPS slots per CTA, one warp each.  W > 1 (what the launcher
// uses): one slot per CTA; warp 0 replays it and the other W-1 warps join it
// for the MT19937 blocks and the tie super-runs.
template <int KM, int W>
__global__ void __launch_bounds__(W == 1 ? 32 * RP_WARPS : 32 * W) k_replay(ReplayArgs A) {
    extern __shared__ __align__(16) unsigned char rp_smem[];
    WarpShared *wsh = reinterpret_cast<WarpShared *>(rp_smem);
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = W == 1 ? blockIdx.x * RP_WARPS + wib : blockIdx.x;
    if (b >= A.nslots) return;
    // only_flagged: the slots the hash select leaves (marginal draws, fewer
    // valid positions than k); every warp of a team leaves together
    if (A.only_flagged && !(A.slots[b].flags & (SLOT_SKIP | SLOT_EMIT_MASKED))) return;
    WarpShared &w = wsh[W == 1 ? wib : 0];
    if constexpr (W > 1) {
        if (wib > 0) {
            team_helper<KM, W>(w);
            return;
        }
    }
    const Slot s = A.slots[b];
    const Geom &g = A.g;
    const int K = s.K;
    const unsigned FULL = 0xffffffffu;

    float cv[KM];
    unsigned cp[KM];
#pragma unroll
    for (int q = 0; q < KM; ++q) { cv[q] = -CUDART_INF_F; cp[q] = 0xffffffffu; }
    unsigned chosen_cell = 0;
    bool have = false;

    if (s.flags & SLOT_SKIP) {
        if (A.state || A.node_cell) {
            // marginal draw over the TI cells (simulation.hpp:586-605; complete TI)
            chosen_cell = unsigned(int(floor((double)__fmul_rn(s.seed, __uint2float_rn((unsigned)A.ti_cells)))));
            // float rounding of seed*cells can reach `cells` only for grids above 2^24 cells
            if ((long long)chosen_cell >= A.ti_cells) chosen_cell = (unsigned)(A.ti_cells - 1);
            if (A.complete_prefix) {
                bool hasNaN = false;
                for (int v = 0; v < A.nvar; ++v) hasNaN |= isnan(A.ti[(long long)chosen_cell * A.nvar + v]);
                if (hasNaN) {
                    // NaN-safe draw (simulation.hpp:616-652): the first cell whose
                    // running count of complete cells reaches floor(seed*(complete/nvar))*nvar
                    const unsigned complete = (unsigned)A.complete_prefix[A.ti_cells - 1];
                    const unsigned pos2 = unsigned(int(floor((double)__fmul_rn(
                                              s.seed, __uint2float_rn(complete / (unsigned)A.nvar))))) *
                                          (unsigned)A.nvar;
                    long long lo2 = 0, hi2 = A.ti_cells;   // first index with prefix >= pos2
                    while (lo2 < hi2) {
                        long long mid = (lo2 + hi2) >> 1;
                        if ((unsigned)A.complete_prefix[mid] < pos2) lo2 = mid + 1;
                        else hi2 = mid;
                    }
                    chosen_cell = (unsigned)(lo2 < A.ti_cells ? lo2 : A.ti_cells - 1);
                }
            }
            have = true;
        }
    } else {
        // generator state: seeded here, or prepared by k_mt_prep together with
        // the blocks that the first masked stretch of the scan skips
        long long preskip = 0;
        if (A.mt_state) {
            // 156 16-byte copies (state rows and w.mt are 16-byte aligned)
            for (int i = lane; i < 156; i += 32) cp_async16(&w.mt[4 * i], A.mt_state + (long long)b * 624 + 4 * i);
            cp_async_wait_all();
            preskip = A.mt_pre[b];
        } else if (lane == 0) {
            mt_seed(w.mt, s.seed);
        }
        __syncwarp();
        int rp = 0, len = 0;
        unsigned cpt = 0;
        long long last = -1;
        const bool emit_masked = (s.flags & (SLOT_EMIT_MASKED | SLOT_MISSING)) != 0;
        const float *rv = A.rec_val + (long long)b * g.nseg * QSK_SEG;
        const int *ri = A.rec_idx + (long long)b * g.nseg * QSK_SEG;
        const int *rc = A.rec_cnt + (long long)b * g.nseg;
        const float *rm = A.rec_max + (long long)b * g.nseg;
        // general replay of one segment's records, 32 per step
        auto general_segment = [&](int sg, int cnt, float smax) {
            const long long base = (long long)sg * QSK_SEG;
            int r0 = 0;
            while (r0 < cnt) {
                const float kth0 = sel_f<KM>(cv, K - 1);
                if (smax < kth0) break;   // nothing left in this segment can enter
                const bool filling = (kth0 == -CUDART_INF_F);
                const int width = filling ? 1 : 32;
                const int j = r0 + lane;
                const bool valid = lane < width && j < cnt;
                const float v = valid ? rv[base + j] : -CUDART_INF_F;
                const int m = valid ? ri[base + j] : 0;
                const unsigned cand = __ballot_sync(FULL, valid && v >= kth0);
                if (cand == 0u) {
                    r0 += width;
                    continue;
                }
                if (filling && !emit_masked) {
                    // masked positions between the previous record and this one are
                    // -inf ties while fewer than K finite values have been seen:
                    // two draws and one cpt increment each, no visible slot change
                    const long long mm = __shfl_sync(FULL, (long long)m, 0);
                    long long c = (mm - (last + 1)) - (valid_prefix(g, s.lo, mm) - valid_prefix(g, s.lo, last + 1));
                    if (c > 0) {
                        // the first skip covers the prepared blocks (c >= the masked
                        // positions before the first valid one, so 2c > preskip)
                        rng_skip<W>(w, lane, rp, len, 2 * c - preskip);
                        preskip = 0;
                        cpt += unsigned(c);
                    }
                }
                rng_ensure<W>(w, lane, rp, len, 64);
                // all K state values equal and nothing above them in the chunk
                if (!filling && sel_f<KM>(cv, 0) == kth0 && __ballot_sync(FULL, valid && v > kth0) == 0) {
                    replay_chunk_ties<KM>(K, valid && v == kth0, m, cp, cpt, rp, w.buf, lane);
                } else if (__popc(cand) <= 4) {
                    replay_scalar<KM>(K, cand, v, m, cv, cp, cpt, rp, w.buf);
                } else {
                    replay_chunk<KM>(K, valid, v, m, cv, cp, cpt, rp, w.buf, lane);
                }
                const unsigned vb = __ballot_sync(FULL, valid);
                last = __shfl_sync(FULL, (long long)m, 31 - __clz(vb));
                r0 += width;
            }
        };
        int sg = 0, wbase = -SEG_WIN;
        while (sg < g.nseg) {
            const float kth_s = sel_f<KM>(cv, K - 1);
            if (kth_s != -CUDART_INF_F) {
                // K finite values: tie super-runs up to the first segment above V
                int xes = 0;
#pragma unroll
                for (int q = 0; q < KM; ++q) xes += (q < K && cv[q] == kth_s) ? 1 : 0;
                sg = replay_tie_stream<KM, W>(K, kth_s, xes, sg, g.nseg, rv, ri, rc, rm, wbase, cp, cpt, rp, len, w,
                                              lane);
                if (sg >= g.nseg) break;
                win_cover(w, wbase, sg, g.nseg, rc, rm, lane);
                general_segment(sg, w.wc[sg - wbase], w.wm[sg - wbase]);
                ++sg;
                continue;
            }
            // general replay, 32 segments at a time, until K finite values are held
            win_cover(w, wbase, sg, g.nseg, rc, rm, lane);
            const int myc = w.wc[sg - wbase + lane];
            const float mym = w.wm[sg - wbase + lane];
            unsigned nz = __ballot_sync(FULL, myc > 0 && mym >= kth_s);
            int next = sg + 32;
            while (nz) {
                const int l = __ffs(nz) - 1;
                nz &= nz - 1;
                general_segment(sg + l, __shfl_sync(FULL, myc, l), __shfl_sync(FULL, mym, l));
                if (sel_f<KM>(cv, K - 1) != -CUDART_INF_F) {
                    next = sg + l + 1;
                    break;
                }
            }
            sg = next;
        }
        // merge loop (quantileSamplingModule.hpp:546-557): repeated first-max extraction
        float fv[KM];
        unsigned fp[KM];
#pragma unroll
        for (int j = 0; j < KM; ++j) {
            fv[j] = -CUDART_INF_F;
            fp[j] = 0xffffffffu;
            if (j < K) {
                int best = 0;
                float bv = cv[0];
#pragma unroll
                for (int l2 = 1; l2 < KM; ++l2)
                    if (l2 < K && cv[l2] > bv) { best = l2; bv = cv[l2]; }
                fv[j] = bv;
                fp[j] = sel_u<KM>(cp, best);
#pragma unroll
                for (int l2 = 0; l2 < KM; ++l2)
                    if (l2 == best) cv[l2] = -CUDART_INF_F;
            }
        }
        // sample(): std::sort by score — insertion sort (stable) for K <= 16
#pragma unroll
        for (int a2 = 1; a2 < KM; ++a2) {
            if (a2 < K) {
#pragma unroll
                for (int c = a2; c > 0; --c) {
                    if (fv[c] > fv[c - 1]) {
                        float tv = fv[c]; fv[c] = fv[c - 1]; fv[c - 1] = tv;
                        unsigned tp = fp[c]; fp[c] = fp[c - 1]; fp[c - 1] = tp;
                    }
                }
            }
        }
        if (lane == 0 && A.out_val) {
#pragma unroll
            for (int j = 0; j < KM; ++j)
                if (j < K) {
                    unsigned out = fp[j];
                    if (A.out_cells) {
                        // cvtIndexToPosition (CPUThreadDevice.cpp:257-268)
                        unsigned position = 0, div = (unsigned)g.N;
                        for (int d = g.nd - 1; d >= 0; --d) {
                            unsigned f = (unsigned)g.fft[d], sr = (unsigned)g.src[d];
                            div /= f;
                            position = position * sr + ((f - (out / div) % f - (unsigned)s.mn[d] - 1u) + sr) % sr;
                        }
                        out = position;
                    }
                    A.out_val[(long long)b * K + j] = fv[j];
                    A.out_pos[(long long)b * K + j] = out;
                }
        }
        if (A.state || A.node_cell) {
            // cvtIndexToPosition (CPUThreadDevice.cpp:257-268), unsigned arithmetic
            unsigned index = sel_u<KM>(fp, s.sel);
            unsigned position = 0;
            unsigned div = (unsigned)g.N;
            for (int d = g.nd - 1; d >= 0; --d) {
                unsigned f = (unsigned)g.fft[d], sr = (unsigned)g.src[d];
                div /= f;
                position = position * sr + ((f - (index / div) % f - (unsigned)s.mn[d] - 1u) + sr) % sr;
            }
            chosen_cell = position;
            have = true;
        }
    }
    if constexpr (W > 1) {
        // the team's work is done (every path of warp 0 reaches this point once)
        __syncwarp();
        if (lane == 0) w.cmd = CMD_EXIT;
        team_bar(32 * W);
    }
    if (lane == 0 && have) {
        if (A.node_cell) A.node_cell[s.node] = chosen_cell;
        if (A.full) {
            // -fs: the node's variable only (simulation.hpp:1016-1024)
            const long long val = (long long)s.cell * A.nvar + s.var;
            if (A.state && isnan(A.state[val])) A.state[val] = A.ti[(long long)chosen_cell * A.nvar + s.var];
            if (A.id_image) A.id_image[val] = chosen_cell * A.nti + A.ti_id;
        } else {
            if (A.state) {
                for (int v = 0; v < A.nvar; ++v) {
                    float *dst = A.state + (long long)s.cell * A.nvar + v;
                    if (isnan(*dst)) *dst = A.ti[(long long)chosen_cell * A.nvar + v];
                }
            }
            if (A.id_image) A.id_image[s.cell] = chosen_cell * A.nti + A.ti_id;
        }
    }
}

// ---------------------------------------------------------------------------
// k best with hash tie-breaks over the map's records (the draw rule of the
// tensor-core form, for the nodes it leaves to the plain map).  Every position
// scoring at least the k-th best is a record (the filter keeps ties), so the
// k largest (score, tie hash) over the records are the k largest over the map.
// One CTA per slot; slots with SLOT_SKIP or SLOT_EMIT_MASKED are left to the
// replay (only_flagged).
// ---------------------------------------------------------------------------
namespace {
template <int W>
__device__ __forceinline__ void hs_insert(unsigned long long (&k)[W], unsigned (&p)[W], unsigned long long key,
                                          unsigned pos) {
    k[0] = key;
    p[0] = pos;
#pragma unroll
    for (int i = 0; i + 1 < W; ++i) {
        const bool sw = k[i] > k[i + 1];
        const unsigned long long a = k[i], c = k[i + 1];
        const unsigned pa = p[i], pc = p[i + 1];
        k[i] = sw ? c : a;
        k[i + 1] = sw ? a : c;
        p[i] = sw ? pc : pa;
        p[i + 1] = sw ? pa : pc;
    }
}
__device__ __forceinline__ unsigned hs_ordered(float f) {
    if (f != f) return 0u;
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
}  // namespace

constexpr int HS_THREADS = 256;
template <int KM>
__global__ void __launch_bounds__(HS_THREADS) k_hash_select(ReplayArgs A) {
    __shared__ unsigned long long sk[HS_THREADS * KM];
    __shared__ unsigned sp[HS_THREADS * KM];
    const int b = blockIdx.x;
    if (b >= A.nslots) return;
    const Slot s = A.slots[b];
    if (s.flags & (SLOT_SKIP | SLOT_EMIT_MASKED)) return;
    const Geom &g = A.g;
    const int K = s.K < KM ? s.K : KM;
    const unsigned seed = __float_as_uint(s.seed) ^ (unsigned(s.node) * 0x85EBCA6Bu);
    unsigned long long rk[KM];
    unsigned rp[KM];
#pragma unroll
    for (int i = 0; i < KM; ++i) {
        rk[i] = 0ull;
        rp[i] = 0u;
    }
    // the thread's K best in rk[KM-K .. KM-1] (ascending array of
    // KM; its minimum rk[0] bounds what may enter)
    const long long base = (long long)b * g.nseg;
    for (int sg = threadIdx.x; sg < g.nseg; sg += HS_THREADS) {
        const int cnt = A.rec_cnt[base + sg];
        if (cnt == 0) continue;
        if (hs_ordered(A.rec_max[base + sg]) < (unsigned)(rk[KM - K] >> 32)) continue;
        const float *rv = A.rec_val + (base + sg) * QSK_SEG;
        const int *ri = A.rec_idx + (base + sg) * QSK_SEG;
        for (int i = 0; i < cnt; ++i) {
            const unsigned idx = (unsigned)ri[i];
            const unsigned long long key = ((unsigned long long)hs_ordered(rv[i]) << 32) | tie_hash(seed, idx);
            if (key > rk[KM - K]) {
                // keep the array's top K: entries below KM-K stay at 0
                hs_insert<KM>(rk, rp, key, idx);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < KM; ++i) {
        sk[i * HS_THREADS + threadIdx.x] = rk[i];
        sp[i * HS_THREADS + threadIdx.x] = rp[i];
    }
    __syncthreads();
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    // K rounds of warp argmax over the block's entries, descending
    unsigned chosen = 0xFFFFFFFFu;
    float cval[KM];
    unsigned cpos[KM];
    int got = 0;
    for (int r = 0; r < K; ++r) {
        unsigned long long bk = 0ull;
        int bi = -1;
        for (int e = lane; e < HS_THREADS * KM; e += 32) {
            const unsigned long long k2 = sk[e];
            if (k2 > bk) {
                bk = k2;
                bi = e;
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
        const unsigned ord = (unsigned)(bk >> 32);
        cval[r] = __uint_as_float((ord & 0x80000000u) ? (ord & 0x7FFFFFFFu) : ~ord);
        cpos[r] = sp[bi];
        __syncwarp();
        if (lane == 0) sk[bi] = 0ull;
        __syncwarp();
        ++got;
    }
    if (lane != 0 || got == 0) return;
    const int sel = s.sel < got ? s.sel : got - 1;
    if (A.out_val)
        for (int j = 0; j < K; ++j) {
            A.out_val[(long long)b * K + j] = j < got ? cval[j] : -CUDART_INF_F;
            A.out_pos[(long long)b * K + j] = j < got ? cpos[j] : 0u;
        }
    // cvtIndexToPosition (CPUThreadDevice.cpp:257-268), unsigned arithmetic
    const unsigned index = cpos[sel];
    unsigned position = 0;
    unsigned div = (unsigned)g.N;
    for (int d = g.nd - 1; d >= 0; --d) {
        unsigned f = (unsigned)g.fft[d], sr = (unsigned)g.src[d];
        div /= f;
        position = position * sr + ((f - (index / div) % f - (unsigned)s.mn[d] - 1u) + sr) % sr;
    }
    chosen = position;
    if (A.drawn_score) {
        A.drawn_score[s.node] = cval[sel];
        A.drawn_scale[s.node] = 0.f;   // the audit's k best come from the same FP32 map: no tolerance
    }
    if (A.node_cell) A.node_cell[s.node] = chosen;
    if (A.state)
        for (int v = 0; v < A.nvar; ++v) {
            float *dst = A.state + (long long)s.cell * A.nvar + v;
            if (isnan(*dst)) *dst = A.ti[(long long)chosen * A.nvar + v];
        }
    if (A.id_image) A.id_image[s.cell] = chosen * A.nti + A.ti_id;
}

// ---------------------------------------------------------------------------
// bit-sliced map for categorical patterns with unit weights
//
// One bit plane per (categorical variable, category) in the flipped scan
// order: bit q of plane (v,c) = [layer_v[q] == c].  For 32 consecutive scan
// positions m0..m0+31 the matches of term t are bits m0-d_t.. of its plane,
// read as one funnel-shifted 32-bit word; an 8-plane bit-sliced counter adds
// them.  With every weight equal to 1 the reference's sum of weights is the
// match count, exact in FP32 (< 2^24), so the scores equal the FP32 map bit
// for bit.  Records, counts and maxima are written in the same 128-position
// segment layout as k_map_records.
// ---------------------------------------------------------------------------
__global__ void k_build_planes(const float *__restrict__ layers, Geom g, int nvar, const int *__restrict__ ncat,
                               const float *__restrict__ catv, int pw, unsigned *__restrict__ planes) {
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long total = (long long)nvar * (QSK_CMAX + 1) * pw;
    if (idx >= total) return;
    const int w = int(idx % pw) - plane_guard(g.N);   // data word (negative: guard)
    int vc = int(idx / pw);
    int c = vc % (QSK_CMAX + 1), v = vc / (QSK_CMAX + 1);
    unsigned word = 0;
    if (w >= 0 && c < ncat[v]) {
        float cv = catv[v * QSK_CMAX + c];
        for (int b = 0; b < 32; ++b) {
            long long q = (long long)w * 32 + b;
            if (q < g.N && layers[(long long)v * g.N + q] == cv) word |= 1u << b;
        }
    }
    planes[idx] = word;
}

// bits [a, b) of a word, 0 <= a, b <= 32
__device__ __forceinline__ unsigned bits_range(int a, int b) {
    if (a >= b) return 0u;
    const unsigned hi = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
    return hi & ~((1u << a) - 1u);
}

// K <= 4: at most 42 registers, 48 warps per SM (measured faster than 48
// registers and 40 warps); the wider top-K states would spill under that cap
template <int KF>
__global__ void __launch_bounds__(256, KF <= 4 ? 6 : 1) k_map_bits(BitArgs A) {
    extern __shared__ int2 bterm[];
    __shared__ Slot ss;
    __shared__ int nbt, s_multi, s_total;
    // staged plane windows of a single-variable slot, per category: lowest and
    // highest word offset of its terms, and where its window starts
    __shared__ int s_lo[QSK_CMAX], s_hi[QSK_CMAX], s_base[QSK_CMAX];
    const int b = blockIdx.y;
    if (threadIdx.x == 0) {
        ss = A.slots[b];
        nbt = 0;
        s_multi = 0;
    }
    if (threadIdx.x < QSK_CMAX) {
        s_lo[threadIdx.x] = INT_MAX;
        s_hi[threadIdx.x] = INT_MIN;
    }
    __syncthreads();
    if (ss.flags & SLOT_SKIP) return;
    const Geom &g = A.g;
    const int seg_begin = blockIdx.x * A.segs_per_cta;
    const int nseg1k = (int)((g.N + 1023) / 1024);
    int seg_end = seg_begin + A.segs_per_cta;
    if (seg_end > nseg1k) seg_end = nseg1k;
    {
        // terms -> (category, word offset), one thread per term; a code that is
        // no category of the TI (or a NaN value) matches nowhere and adds
        // nothing to the counts, so the term is dropped (the count is a sum of
        // 0/1 matches: its order is free)
        const Term *src = A.terms + (long long)b * A.maxterms;
        const StaticTerm *ssrc = A.sterms ? A.sterms + (long long)b * A.maxterms : nullptr;
        const int N32 = (int)g.N;
        for (int t = threadIdx.x; t < ss.nterms; t += blockDim.x) {
            int base;
            float val;
            if (ssrc) {
                const StaticTerm st = ssrc[t];
                base = st.base;
                val = st.src >= 0 ? A.state[st.src] : A.init[-(long long)st.src - 1];
            } else {
                const Term tm = src[t];
                base = tm.base;
                val = tm.b;
            }
            // base = v*N - d with 0 <= d < N
            const int v = base > 0 ? (base + N32 - 1) / N32 : 0;
            const int d = v * N32 - base;
            int c = QSK_CMAX;
            const int nc = A.ncat[v];
            for (int q = 0; q < nc; ++q)
                if (A.catv[v * QSK_CMAX + q] == val) { c = q; break; }
            if (c == QSK_CMAX) continue;
            // positions 32k..32k+31 read source bits from word k + floor(-d/32),
            // shifted right by (-d) mod 32
            const int off = plane_guard(g.N) + ((-d) >> 5);
            const int o = atomicAdd(&nbt, 1);
            if (v > 0) {
                s_multi = 1;
                bterm[o] = make_int2((v * (QSK_CMAX + 1) + c) * A.pw + off, (-d) & 31);
            } else {
                atomicMin(&s_lo[c], off);
                atomicMax(&s_hi[c], off);
                bterm[o] = make_int2(c * A.pw + off, ((-d) & 31) | (c << 8));
            }
        }
        if (threadIdx.x == 0 && ssrc && A.no_verbatim && ss.vtpl >= 0)
            ss.excl = verbatim_excl(g, A.tpl + ss.vtpl * g.nd, A.id_image[ss.vcell], ss.mn);
    }
    __syncthreads();
    const int nt = nbt;
    // Staging: the words of each category plane that this CTA's segments read
    // ([lo + 32*seg_begin, hi + 32*seg_end + 1)) go to shared memory, where a
    // warp's 32 consecutive words are one conflict-free access at any word
    // alignment (from global memory they span two cache lines).
    unsigned *stage = reinterpret_cast<unsigned *>(bterm + A.maxterms);
    if (threadIdx.x < 32) {
        const int c = threadIdx.x;
        const int len = s_lo[c] <= s_hi[c] ? s_hi[c] - s_lo[c] + 32 * (seg_end - seg_begin) + 1 : 0;
        int inc = len;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, off);
            if (c >= off) inc += y;
        }
        s_base[c] = inc - len;
        if (c == 31) s_total = inc;
    }
    __syncthreads();
    const bool staged = !s_multi && s_total <= A.stage_words && A.stage_words > 0;
    if (staged) {
        for (int c = 0; c < QSK_CMAX; ++c) {
            if (s_lo[c] > s_hi[c]) continue;
            const int len = s_hi[c] - s_lo[c] + 32 * (seg_end - seg_begin) + 1;
            const unsigned *src = A.planes + (long long)c * A.pw + s_lo[c] + 32 * seg_begin;
            unsigned *dst = stage + s_base[c];
            for (int w = threadIdx.x; w < len; w += blockDim.x) dst[w] = __ldg(src + w);
        }
        for (int t = threadIdx.x; t < nt; t += blockDim.x) {
            const int2 bt = bterm[t];
            const int c = bt.y >> 8;
            const int off = bt.x - c * A.pw;
            bterm[t] = make_int2(s_base[c] + off - s_lo[c] - 32 * seg_begin, bt.y & 31);
        }
    } else {
        for (int t = threadIdx.x; t < nt; t += blockDim.x) bterm[t].y &= 31;
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    const bool emit_masked = (ss.flags & SLOT_EMIT_MASKED) != 0;
    float *rv = A.rec_val + (long long)b * g.nseg * QSK_SEG;
    int *ri = A.rec_idx + (long long)b * g.nseg * QSK_SEG;

    for (int sg = seg_begin + warp; sg < seg_end; sg += nwarps) {
        const long long m0 = (long long)sg * 1024 + 32 * lane;
        // validity of the lane's 32 positions
        unsigned vmask = 0, emask = 0;
        if (m0 < g.N && g.fft[0] >= 32) {
            // the 32 positions lie in at most two rows of the x dimension
            const long long rem = g.N - m0;
            emask = rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
            // scan indices are below 2^31: 32-bit digits (row r holds digits 1..)
            const unsigned X = (unsigned)g.fft[0];
            const unsigned r0 = (unsigned)m0 / X;
            const int x0 = int((unsigned)m0 - r0 * X);
            auto row_ok = [&](unsigned r) {
                bool ok = true;
#pragma unroll
                for (int d = 1; d < QSK_MAXD; ++d)
                    if (d < g.nd) {
                        const unsigned f = (unsigned)g.fft[d];
                        ok &= int(r % f) >= ss.lo[d];
                        r /= f;
                    }
                return ok;
            };
            auto range = [](int a, int b) -> unsigned {   // bits [a, b), 0 <= a, b <= 32
                if (a >= b) return 0u;
                const unsigned hi = b >= 32 ? 0xffffffffu : ((1u << b) - 1u);
                return hi & ~((1u << a) - 1u);
            };
            const int first = X - x0;   // positions p < first are in row r0
            unsigned m = 0;
            if (row_ok(r0)) m |= range(max(0, ss.lo[0] - x0), min(32, first));
            if (first < 32 && row_ok(r0 + 1)) m |= range(min(32, first + ss.lo[0]), 32);
            vmask = m & emask;
        } else if (m0 < g.N) {
            // narrow x dimension: incremental digits
            int dig[QSK_MAXD];
#pragma unroll
            for (int d = 0; d < QSK_MAXD; ++d)
                dig[d] = d < g.nd ? int(((unsigned)m0 / (unsigned)g.sstride[d]) % (unsigned)g.fft[d]) : 0;
            bool rowok = true;
#pragma unroll
            for (int d = 1; d < QSK_MAXD; ++d)
                if (d < g.nd) rowok &= dig[d] >= ss.lo[d];
            for (int bit = 0; bit < 32; ++bit) {
                if (m0 + bit >= g.N) break;
                emask |= 1u << bit;
                if (rowok && dig[0] >= ss.lo[0]) vmask |= 1u << bit;
                if (++dig[0] == g.fft[0]) {
                    dig[0] = 0;
                    for (int d = 1; d < g.nd; ++d) {
                        if (++dig[d] < g.fft[d]) break;
                        dig[d] = 0;
                    }
                    rowok = true;
                    for (int d = 1; d < g.nd; ++d) rowok &= dig[d] >= ss.lo[d];
                }
            }
        }
        // bit-sliced counter: c0 (ones), c1 (twos), c2 (fours), c3 (eights)
        // fed by carry-save adders (Harley-Seal) over groups of 16 match
        // words, c4..c7 count sixteens; a tail of 8 and single words ripples
        unsigned c0 = 0, c1 = 0, c2 = 0, c3 = 0, c4 = 0, c5 = 0, c6 = 0, c7 = 0;
        if (vmask) {
            const int mw = int(m0) >> 5;
            auto count = [&](auto match) {
                auto csa = [](unsigned &h, unsigned &l, unsigned a, unsigned b, unsigned c) {
                    const unsigned u = a ^ b;
                    h = (a & b) | (u & c);
                    l = u ^ c;
                };
                int t = 0;
                for (; t + 16 <= nt; t += 16) {
                    unsigned twosA, twosB, foursA, foursB, eightsA, eightsB, sixteens;
                    csa(twosA, c0, c0, match(t), match(t + 1));
                    csa(twosB, c0, c0, match(t + 2), match(t + 3));
                    csa(foursA, c1, c1, twosA, twosB);
                    csa(twosA, c0, c0, match(t + 4), match(t + 5));
                    csa(twosB, c0, c0, match(t + 6), match(t + 7));
                    csa(foursB, c1, c1, twosA, twosB);
                    csa(eightsA, c2, c2, foursA, foursB);
                    csa(twosA, c0, c0, match(t + 8), match(t + 9));
                    csa(twosB, c0, c0, match(t + 10), match(t + 11));
                    csa(foursA, c1, c1, twosA, twosB);
                    csa(twosA, c0, c0, match(t + 12), match(t + 13));
                    csa(twosB, c0, c0, match(t + 14), match(t + 15));
                    csa(foursB, c1, c1, twosA, twosB);
                    csa(eightsB, c2, c2, foursA, foursB);
                    csa(sixteens, c3, c3, eightsA, eightsB);
                    unsigned x = sixteens, t0;
                    t0 = c4 & x; c4 ^= x; x = t0;
                    t0 = c5 & x; c5 ^= x; x = t0;
                    t0 = c6 & x; c6 ^= x; x = t0;
                    c7 ^= x;
                }
                for (; t + 8 <= nt; t += 8) {
                    unsigned twosA, twosB, foursA, foursB, eights;
                    csa(twosA, c0, c0, match(t), match(t + 1));
                    csa(twosB, c0, c0, match(t + 2), match(t + 3));
                    csa(foursA, c1, c1, twosA, twosB);
                    csa(twosA, c0, c0, match(t + 4), match(t + 5));
                    csa(twosB, c0, c0, match(t + 6), match(t + 7));
                    csa(foursB, c1, c1, twosA, twosB);
                    csa(eights, c2, c2, foursA, foursB);
                    unsigned x = eights, t0;
                    t0 = c3 & x; c3 ^= x; x = t0;
                    t0 = c4 & x; c4 ^= x; x = t0;
                    t0 = c5 & x; c5 ^= x; x = t0;
                    t0 = c6 & x; c6 ^= x; x = t0;
                    c7 ^= x;
                }
                for (; t < nt; ++t) {
                    unsigned x = match(t), t0;
                    t0 = c0 & x; c0 ^= x; x = t0;
                    t0 = c1 & x; c1 ^= x; x = t0;
                    t0 = c2 & x; c2 ^= x; x = t0;
                    t0 = c3 & x; c3 ^= x; x = t0;
                    t0 = c4 & x; c4 ^= x; x = t0;
                    t0 = c5 & x; c5 ^= x; x = t0;
                    t0 = c6 & x; c6 ^= x; x = t0;
                    c7 ^= x;
                }
            };
            if (staged) {
                const unsigned *S = stage + mw;
                count([&](int t) -> unsigned {
                    const int2 bt = bterm[t];
                    return __funnelshift_r(S[bt.x], S[bt.x + 1], unsigned(bt.y));
                });
            } else {
                const unsigned *P = A.planes + mw;
                count([&](int t) -> unsigned {
                    const int2 bt = bterm[t];
                    return __funnelshift_r(__ldg(P + bt.x), __ldg(P + bt.x + 1), unsigned(bt.y));
                });
            }
        }
        // Scores stay bit-sliced: position p of the lane holds the count
        // sum_b ((c_b >> p) & 1) << b where it is valid and not excluded, -inf
        // elsewhere.  Lane top-K by repeated bit-sliced maximum extraction.
        unsigned vm = vmask;
        if (ss.excl >= 0 && (long long)ss.excl >= m0 && (long long)ss.excl < m0 + 32)
            vm &= ~(1u << unsigned(ss.excl - m0));
        auto count_at = [&](int p) -> int {
            return int(((c0 >> p) & 1u) | (((c1 >> p) & 1u) << 1) | (((c2 >> p) & 1u) << 2) |
                       (((c3 >> p) & 1u) << 3) | (((c4 >> p) & 1u) << 4) | (((c5 >> p) & 1u) << 5) |
                       (((c6 >> p) & 1u) << 6) | (((c7 >> p) & 1u) << 7));
        };
        float lst[KF];
#pragma unroll
        for (int q = 0; q < KF; ++q) lst[q] = -CUDART_INF_F;
        float lmax = -CUDART_INF_F;
        {
            unsigned rest = vm;
            int filled = 0;
            for (int q = 0; q < KF && rest != 0u && filled < KF; ++q) {
                unsigned cand = rest;
                int val = 0;
                const unsigned cb[8] = {c0, c1, c2, c3, c4, c5, c6, c7};
#pragma unroll
                for (int bb = 7; bb >= 0; --bb) {
                    const unsigned t = cand & cb[bb];
                    if (t) {
                        cand = t;
                        val |= 1 << bb;
                    }
                }
                const int mult = __popc(cand);
                const float fv = (float)val;
#pragma unroll
                for (int q2 = 0; q2 < KF; ++q2)
                    if (q2 >= filled && q2 < filled + mult) lst[q2] = fv;
                if (q == 0) lmax = fv;
                filled += mult;
                rest &= ~cand;
            }
        }
        // exclusive prefix of the lane states across the 1024-position segment
        float inc[KF];
#pragma unroll
        for (int q = 0; q < KF; ++q) inc[q] = lst[q];
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            float rcv[KF], mrg[KF];
#pragma unroll
            for (int q = 0; q < KF; ++q) rcv[q] = __shfl_up_sync(0xffffffffu, inc[q], off);
            if (lane >= off) {
                topk_merge<KF>(inc, rcv, mrg);
#pragma unroll
                for (int q = 0; q < KF; ++q) inc[q] = mrg[q];
            }
        }
        float st[KF];
#pragma unroll
        for (int q = 0; q < KF; ++q) {
            float y = __shfl_up_sync(0xffffffffu, inc[q], 1);
            st[q] = lane == 0 ? -CUDART_INF_F : y;
        }
        // Lane 0 has no earlier lane, so its running K-th starts from nothing
        // and most of its positions would be visited one by one below.  The
        // warp decides them instead: position p of lane 0 on lane p, and an
        // exclusive prefix top-K over the lanes gives the K-th before each.
        float x0v;
        unsigned rmask0;
        {
            const unsigned vm0 = __shfl_sync(0xffffffffu, vm, 0);
            const unsigned recok0 = __shfl_sync(0xffffffffu, emit_masked ? emask : (emask & vmask), 0);
            const unsigned cnt = ((__shfl_sync(0xffffffffu, c0, 0) >> lane) & 1u) |
                                 (((__shfl_sync(0xffffffffu, c1, 0) >> lane) & 1u) << 1) |
                                 (((__shfl_sync(0xffffffffu, c2, 0) >> lane) & 1u) << 2) |
                                 (((__shfl_sync(0xffffffffu, c3, 0) >> lane) & 1u) << 3) |
                                 (((__shfl_sync(0xffffffffu, c4, 0) >> lane) & 1u) << 4) |
                                 (((__shfl_sync(0xffffffffu, c5, 0) >> lane) & 1u) << 5) |
                                 (((__shfl_sync(0xffffffffu, c6, 0) >> lane) & 1u) << 6) |
                                 (((__shfl_sync(0xffffffffu, c7, 0) >> lane) & 1u) << 7);
            const bool val = (vm0 >> lane) & 1u;
            x0v = val ? (float)cnt : -CUDART_INF_F;
            float in0[KF];
            in0[0] = x0v;
#pragma unroll
            for (int q = 1; q < KF; ++q) in0[q] = -CUDART_INF_F;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                float rcv[KF], mrg[KF];
#pragma unroll
                for (int q = 0; q < KF; ++q) rcv[q] = __shfl_up_sync(0xffffffffu, in0[q], off);
                if (lane >= off) {
                    topk_merge<KF>(in0, rcv, mrg);
#pragma unroll
                    for (int q = 0; q < KF; ++q) in0[q] = mrg[q];
                }
            }
            const float y = __shfl_up_sync(0xffffffffu, in0[KF - 1], 1);
            const float kth = lane == 0 ? -CUDART_INF_F : y;
            // before K finite values every position that can be a candidate is
            // a record; afterwards the valid ones not below the K-th
            const bool rec = kth == -CUDART_INF_F ? ((recok0 >> lane) & 1u) != 0u : (val && x0v >= kth);
            rmask0 = __ballot_sync(0xffffffffu, rec);
        }
        // record flags: value not below the K-th best of everything before it
        // (earlier lanes, then earlier positions of this lane)
        unsigned rmask = lane == 0 ? rmask0 : 0u;
        const float T0s = st[KF - 1];
        unsigned eqm = 0u;       // records whose value is tval (no count extraction)
        float tval = 0.f;
        unsigned from = lane == 0 ? 0u : 0xffffffffu;   // positions decided by the threshold path below
        float T0 = T0s;
        if (lane != 0 && T0 == -CUDART_INF_F) {
            // Fewer than K finite values before this lane: every position is a
            // record until K finite values are held (masked ones only when they
            // can be candidates).  Only the valid positions up to that point are
            // visited one by one; the rest of the lane takes the threshold path.
            const unsigned recok = emit_masked ? emask : (emask & vmask);
            unsigned vv = vm;
            int cur = 0;
            while (vv && st[KF - 1] == -CUDART_INF_F) {
                const int bit = __ffs(vv) - 1;
                vv &= vv - 1u;
                rmask |= recok & bits_range(cur, bit);
                rmask |= 1u << bit;
                topk_insert<KF>(st, (float)count_at(bit));
                cur = bit + 1;
            }
            if (st[KF - 1] == -CUDART_INF_F) {
                rmask |= recok & bits_range(cur, 32);
                from = 0u;
            } else {
                from = bits_range(cur, 32);
            }
            T0 = st[KF - 1];
        }
        if (from) {
            // only positions with count >= T0 can be records (the running K-th
            // never drops below T0; a smaller value leaves the state unchanged)
            const int T = (int)T0;
            unsigned gt = 0u, eq = vm;
            const unsigned cb[8] = {c0, c1, c2, c3, c4, c5, c6, c7};
#pragma unroll
            for (int bb = 7; bb >= 0; --bb) {
                if ((T >> bb) & 1) {
                    eq &= cb[bb];
                } else {
                    gt |= eq & cb[bb];
                    eq &= ~cb[bb];
                }
            }
            if (T > 255) gt = eq = 0u;
            gt &= from;
            eq &= from;
            // Positions equal to T0 are records while the running K-th is still
            // T0 and never change the state; only positions above T0 need their
            // count and an insertion.  The first insertion that lifts the K-th
            // above T0 ends the equal records.
            unsigned eqcut = 0xffffffffu;
            unsigned g = gt;
            while (g) {
                const int bit = __ffs(g) - 1;
                g &= g - 1u;
                const float x = (float)count_at(bit);
                if (x >= st[KF - 1]) rmask |= 1u << bit;
                topk_insert<KF>(st, x);
                if (eqcut == 0xffffffffu && st[KF - 1] > T0) eqcut = bit >= 31 ? 0xffffffffu : ((2u << bit) - 1u);
            }
            rmask |= eq & eqcut;
            eqm = eq;
            tval = T0;
        }
        // offsets inside each 128-position sub-segment (4 lanes)
        const int rc = __popc(rmask);
        int pre = rc;
        int y1 = __shfl_up_sync(0xffffffffu, pre, 1);
        if ((lane & 3) >= 1) pre += y1;
        int y2 = __shfl_up_sync(0xffffffffu, pre, 2);
        if ((lane & 3) >= 2) pre += y2;
        const int excl = pre - rc;
        const int tot = __shfl_sync(0xffffffffu, pre, (lane | 3));
        float gmax = lmax;
        gmax = fmaxf(gmax, __shfl_xor_sync(0xffffffffu, gmax, 1));
        gmax = fmaxf(gmax, __shfl_xor_sync(0xffffffffu, gmax, 2));
        const long long sub = (long long)sg * 8 + (lane >> 2);
        // lane 0's records, one per lane (the first ones of its sub-segment)
        if ((rmask0 >> lane) & 1u) {
            const long long r0 = (long long)sg * 8 * QSK_SEG + __popc(rmask0 & lanemask_lt());
            rv[r0] = x0v;
            ri[r0] = int((long long)sg * 1024 + lane);
        }
        if (sub < g.nseg) {
            const long long rb = sub * QSK_SEG + excl;
            int o = 0;
            unsigned rm = lane == 0 ? 0u : rmask;
            while (rm) {
                const int bit = __ffs(rm) - 1;
                rm &= rm - 1u;
                rv[rb + o] = ((eqm >> bit) & 1u) ? tval : (((vm >> bit) & 1u) ? (float)count_at(bit) : -CUDART_INF_F);
                ri[rb + o] = int(m0 + bit);
                o++;
            }
            if ((lane & 3) == 0) {
                A.rec_cnt[(long long)b * g.nseg + sub] = tot;
                A.rec_max[(long long)b * g.nseg + sub] = gmax;
            }
        }
    }
}

// The slot of path node i and its terms without their values (bit-sliced
// simulations: unit weights, categorical variables, complete TI): everything
// k_prep_sim derives from the neighbour lists, computed one batch ahead.
// The map reads the values (and derives the -nV exclusion) when it runs.
__device__ void write_static_slot(const SimPrepArgs &A, int b, int i, unsigned pv, unsigned cell, const NodeGeom &ng,
                                  int lane) {
    const int cnt = A.nb_count[i];
    const int nd = A.g.nd;
    Slot s;
    s.node = i;
    s.cell = cell;
    s.var = A.full ? int(pv % unsigned(A.nvar)) : 0;
    s.seed = A.seeds[i];
    s.K = ng.Ki;
    s.sel = selected_index(s.seed, ng.lk, A.nti);
    if (s.sel < 0) s.sel = 0;
    if (s.sel > ng.Ki - 1) s.sel = ng.Ki - 1;
    s.flags = 0;
    s.nterms = 0;
    s.excl = -1;
    s.cmask_base = 0;
    s.vcell = 0;
    s.vtpl = -1;
#pragma unroll
    for (int d = 0; d < QSK_MAXD; ++d) {
        s.mn[d] = ng.mn[d];
        s.lo[d] = ng.lo[d];
    }
    if (ng.skip) {
        s.flags |= SLOT_SKIP;
    } else {
        if (ng.nvalid < ng.Ki) s.flags |= SLOT_EMIT_MASKED;
        int base_out = 0;
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            const int j = j0 + lane;
            StaticTerm tl[4];
            int nt = 0;
            if (j < cnt) {
                const int t = A.nb_tpl[(long long)i * A.n + j];
                const unsigned nc = A.nb_cell[(long long)i * A.n + j];
                long long d_flat = 0;
                for (int d = 0; d < nd; ++d) d_flat += (long long)(A.tpl[t * nd + d] - ng.mn[d]) * A.g.sstride[d];
                for (int v = 0; v < A.nvar && v < 4; ++v) {
                    if (A.full) {
                        if (!((A.nb_mask[(long long)i * A.n + j] >> v) & 1u)) continue;
                    } else if (A.node_nv && j >= A.node_nv[(long long)i * A.nvar + v]) {
                        continue;
                    }
                    if (A.wtab[t * A.nvar + v] == 0.f) continue;
                    const long long sidx = (long long)nc * A.nvar + v;
                    StaticTerm st;
                    st.base = int((long long)v * A.g.N - d_flat);
                    st.src = (nc == cell && !A.full) ? int(-sidx - 1) : int(sidx);
                    tl[nt++] = st;
                }
            }
            int incl = nt;
            for (int off = 1; off < 32; off <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += y;
            }
            const int excl = incl - nt;
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            for (int q = 0; q < nt; ++q) {
                const int o = base_out + excl + q;
                if (o < A.maxterms) A.sterms[(long long)b * A.maxterms + o] = tl[q];
            }
            base_out += total;
        }
        if (base_out > A.maxterms) {
            if (lane == 0) atomicExch(A.status, DEV_TOO_MANY_TERMS);
            base_out = A.maxterms;
        }
        s.nterms = base_out;
        if (A.no_verbatim && cnt > 1 && !A.full) {
            s.vtpl = A.nb_tpl[(long long)i * A.n + 1];
            s.vcell = A.nb_cell[(long long)i * A.n + 1];
        }
    }
    if (lane == 0) A.slots[b] = s;
}

// MT19937 state of each slot ahead of its replay (one warp per slot; the
// host runs it for the next batch while the current one is simulated, as it
// reads the neighbour lists only): the seeding and, with masked positions
// not emitted as records, the state-only blocks of the replay's first
// skip.  That skip covers the c
// masked positions before the first record (two draws each); c is at least
// the number c0 of masked positions before the first valid one, so the
// blocks that rng_skip regenerates without output for 2*c0 draws,
// (2*c0 - 1) / 624 of them, are the first blocks of the real skip too.
__global__ void __launch_bounds__(32 * RP_WARPS) k_mt_prep(SimPrepArgs A, unsigned *__restrict__ state,
                                                           int *__restrict__ pre) {
    __shared__ unsigned mt[RP_WARPS][624 + 32];
    __shared__ float dummy[RP_WARPS][32];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * RP_WARPS + wib;
    if (b >= A.nslots) return;
    const int i = A.nodes[b];
    const unsigned pv = A.path[A.begin + i];
    const unsigned cell = A.full ? pv / unsigned(A.nvar) : pv;
    const NodeGeom ng = node_geometry(A, i, cell, lane);
    if (A.sterms) write_static_slot(A, b, i, pv, cell, ng, lane);
    if (ng.skip) return;
    if (lane == 0) mt_seed(mt[wib], A.seeds[i]);
    __syncwarp();
    int blocks = 0;
    const Geom &g = A.g;
    if (ng.nvalid >= ng.Ki && !A.missing && ng.nvalid > 0) {
        long long m0 = 0;
        for (int d = 0; d < g.nd; ++d) m0 += (long long)ng.lo[d] * g.sstride[d];
        const long long n = 2 * (m0 - valid_prefix(g, ng.lo, m0));
        if (n > 624) blocks = int((n - 1) / 624);
    }
    for (int t = 0; t < blocks; ++t) mt_twist<false>(mt[wib], lane, nullptr, dummy[wib]);
    __syncwarp();
    for (int i = lane; i < 624; i += 32) state[(long long)b * 624 + i] = mt[wib][i];
    if (lane == 0) pre[b] = 624 * blocks;
}

// Verbatim exclusion with a radius (CPUThreadDevice::setValueInErrorArrayWithRadius,
// G2S src/CPUThreadDevice.cpp:310-342): from the scan index c, level L = nd..2
// steps i_L in [-r, r] with r = ceil(sqrt(R2 - d2)) by fft[L-1] (d2 the sum of
// the squares of the outer steps, a level entered only while d2 <= R2), and
// level 1 steps by fft[0], marking (c + offset + N) mod N in 32-bit unsigned
// arithmetic as the reference does.  One CTA per slot: the outer steps are a
// box [-R, R]^(nd-1) enumerated by the threads, each thread runs the level-1
// loop of its tuples.
__global__ void k_radius_mask(const int *__restrict__ center, const float *__restrict__ radius, Geom g,
                              unsigned *__restrict__ mask, long long xwords) {
    const int b = blockIdx.x;
    unsigned *xm = mask + (long long)b * xwords;
    for (long long q = threadIdx.x; q < xwords; q += blockDim.x) xm[q] = 0u;
    __syncthreads();
    const int c = center[b];
    const float rad = radius[b];
    if (c < 0 || !(rad >= 1.f)) return;
    const float R2 = rad * rad;
    const int R = int(ceil(sqrt((double)R2)));
    const unsigned s = (unsigned)g.N;
    const int nouter = g.nd - 1;
    long long box = 1;
    for (int L = 0; L < nouter; ++L) box *= 2 * R + 1;
    for (long long t = threadIdx.x; t < box; t += blockDim.x) {
        // outer tuple (i_nd, ..., i_2), outermost first
        long long rest = t;
        unsigned pos = (unsigned)c;
        unsigned d2 = 0;
        bool ok = true;
        for (int L = g.nd; L >= 2 && ok; --L) {
            const int i = int(rest % (2 * R + 1)) - R;
            rest /= (2 * R + 1);
            // level L is entered with d2 <= R2 and runs i in [-r, r]
            if (!((float)d2 <= R2)) { ok = false; break; }
            const int r = int(ceil(sqrt((double)(R2 - (float)d2))));
            if (i < -r || i > r) { ok = false; break; }
            pos += (unsigned)(i * (int)g.fft[L - 1]);
            d2 += (unsigned)(i * i);
        }
        if (!ok || !((float)d2 <= R2)) continue;
        const int r1 = int(ceil(sqrt((double)(R2 - (float)d2))));
        for (int i = -r1; i <= r1; ++i) {
            const unsigned m = (pos + (unsigned)(i * (int)g.fft[0]) + s) % s;
            atomicOr(xm + (m >> 5), 1u << (m & 31));
        }
    }
}

// ---------------------------------------------------------------------------
// launch wrappers (called by the host engine)
// ---------------------------------------------------------------------------
cudaError_t launch_build_layers(const float *ti, int nvar, const int *types, const Geom &g, float *layers, int missing,
                                cudaStream_t st) {
    long long blocks = (g.N + 255) / 256;
    k_build_layers<<<(unsigned)blocks, 256, 0, st>>>(ti, nvar, types, g, layers, missing);
    return cudaGetLastError();
}

cudaError_t launch_neighbours(const GridDesc &dg, const int *tpl, int ntpl, const unsigned *path, unsigned begin,
                              long long nodes, const unsigned *posterior, int n, int *nb_count, int *nb_tpl,
                              unsigned *nb_cell, const int *node_kernel, const int *tpl_range, const int *node_lim,
                              cudaStream_t st) {
    if (nodes <= 0) return cudaSuccess;
    k_neighbours<<<(unsigned)((nodes * 32 + 255) / 256), 256, 0, st>>>(dg, tpl, ntpl, path, begin, nodes, posterior, n,
                                                                       nb_count, nb_tpl, nb_cell, node_kernel,
                                                                       tpl_range, node_lim);
    return cudaGetLastError();
}

cudaError_t launch_neighbours_full(const GridDesc &dg, const int *tpl, int ntpl, const unsigned *path, unsigned begin,
                                   long long nodes, const unsigned *posterior, int nvar, int n, const int *node_nv,
                                   int *nb_count, int *nb_tpl, unsigned *nb_cell, unsigned char *nb_mask,
                                   const int *node_kernel, const int *tpl_range, cudaStream_t st) {
    if (nodes <= 0) return cudaSuccess;
    k_neighbours_full<<<(unsigned)((nodes * 32 + 255) / 256), 256, 0, st>>>(dg, tpl, ntpl, path, begin, nodes, posterior,
                                                                            nvar, n, node_nv, nb_count, nb_tpl, nb_cell,
                                                                            nb_mask, node_kernel, tpl_range);
    return cudaGetLastError();
}

cudaError_t launch_levels(const LevelArgs &a, cudaStream_t st) {
    long long nodes = a.nodes;
    if (nodes <= 0) return cudaSuccess;
    const unsigned nb = (unsigned)((nodes + 255) / 256);
    const long long ntiles = (nodes + 1023) / 1024;
    cudaError_t e;
    if ((e = cudaMemsetAsync(a.level, 0xff, sizeof(int) * size_t(nodes), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.cnt, 0, sizeof(int) * size_t(nodes + 2), st)) != cudaSuccess) return e;
    int dev = 0, sms = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    long long blocks = (long long)sms * 8;
    const long long need = (nodes * 32 + 255) / 256;
    if (blocks > need) blocks = need;
    k_level_flow<<<(unsigned)blocks, 256, 0, st>>>(nodes, a.n, a.nb_count, a.nb_cell, a.nb_mask, a.nvar, a.node_of_cell,
                                                   a.level, a.cnt + nodes + 1, a.nl_out, a.status,
                                                   a.spin_limit ? a.spin_limit : (1u << 22), a.hold);
    k_level_count<<<nb, 256, 0, st>>>(nodes, a.level, a.cnt);
    k_scan_tiles<<<(unsigned)ntiles, 1024, 0, st>>>(nodes, a.cnt, a.start, a.tile_sum);
    k_scan_sums<<<1, 32, 0, st>>>((int)ntiles, a.tile_sum);
    k_scan_add<<<(unsigned)((nodes + 1 + 255) / 256), 256, 0, st>>>(nodes, a.start, a.cursor, a.tile_sum);
    k_level_scatter<<<nb, 256, 0, st>>>(nodes, a.level, a.cursor, a.level_nodes);
    return cudaGetLastError();
}

cudaError_t launch_prep_tc_nodes(const SimPrepArgs &p, const TcNodeArgs &a, cudaStream_t st) {
    if (!a.A || a.nslots != p.nslots || a.rows < a.nslots || (a.Kp * (a.fmt == 1 ? 1 : 2)) % 16 != 0)
        return cudaErrorInvalidValue;
    const long long prep_blocks = ((long long)p.nslots * 32 + 255) / 256;
    const long long node_blocks = (a.rows * 32 + 255) / 256;
    k_prep_tc_nodes<<<(unsigned)(prep_blocks + node_blocks), 256, 0, st>>>(p, a, (unsigned)prep_blocks);
    return cudaGetLastError();
}

cudaError_t launch_prep_sim(const SimPrepArgs &a, cudaStream_t st) {
    int threads = 256;
    long long blocks = ((long long)a.nslots * 32 + threads - 1) / threads;
    k_prep_sim<<<(unsigned)blocks, threads, 0, st>>>(a);
    return cudaGetLastError();
}

int map_segs_per_cta(const Geom &g, int nslots) {
    // enough CTAs to fill the GPU several times over, at most 32 segments each
    long long target = 148LL * 8;
    long long per = ((long long)g.nseg * nslots + target - 1) / target;
    if (per < 8) per = 8;
    if (per > 32) per = 32;
    return (int)per;
}

cudaError_t launch_map_records(const MapArgs &a, int nslots, int K, int maxterms_in_batch, cudaStream_t st) {
    int threads = 256;
    dim3 grid((unsigned)((a.g.nseg + a.segs_per_cta - 1) / a.segs_per_cta), (unsigned)nslots);
    size_t smem = sizeof(Term) * (size_t)(maxterms_in_batch > 0 ? maxterms_in_batch : 1);
    if (K <= 1) k_map_records<1><<<grid, threads, smem, st>>>(a);
    else if (K <= 2) k_map_records<2><<<grid, threads, smem, st>>>(a);
    else if (K <= 4) k_map_records<4><<<grid, threads, smem, st>>>(a);
    else if (K <= 8) k_map_records<8><<<grid, threads, smem, st>>>(a);
    else k_map_records<16><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_build_planes(const float *layers, const Geom &g, int nvar, const int *ncat, const float *catv,
                                int pw, unsigned *planes, cudaStream_t st) {
    long long total = (long long)nvar * (QSK_CMAX + 1) * pw;
    k_build_planes<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(layers, g, nvar, ncat, catv, pw, planes);
    return cudaGetLastError();
}

// shared-memory words for the staged plane windows of k_map_bits (24 KB)
#define MAP_BITS_STAGE_WORDS 6144

int map_bits_segs_per_cta(const Geom &g, int nslots) {
    long long nseg1k = (g.N + 1023) / 1024;
    long long target = 148LL * 8;
    long long per = (nseg1k * nslots + target - 1) / target;
    if (per < 8) per = 8;
    if (per > 16) per = 16;
    return (int)per;
}

cudaError_t launch_map_bits(const BitArgs &args, int nslots, int K, int maxterms_in_batch, cudaStream_t st) {
    int threads = 256;
    BitArgs a = args;
    if (a.maxterms < maxterms_in_batch) return cudaErrorInvalidValue;
    a.stage_words = MAP_BITS_STAGE_WORDS;
    long long nseg1k = (a.g.N + 1023) / 1024;
    dim3 grid((unsigned)((nseg1k + a.segs_per_cta - 1) / a.segs_per_cta), (unsigned)nslots);
    size_t smem = sizeof(int2) * (size_t)(a.maxterms > 0 ? a.maxterms : 1) + sizeof(unsigned) * (size_t)a.stage_words;
    if (K <= 1) k_map_bits<1><<<grid, threads, smem, st>>>(a);
    else if (K <= 2) k_map_bits<2><<<grid, threads, smem, st>>>(a);
    else if (K <= 4) k_map_bits<4><<<grid, threads, smem, st>>>(a);
    else if (K <= 8) k_map_bits<8><<<grid, threads, smem, st>>>(a);
    else k_map_bits<16><<<grid, threads, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t set_map_smem_limit(int bytes) {
    cudaError_t e = cudaSuccess;
    e = cudaFuncSetAttribute(k_map_records<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_map_records<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_map_records<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_map_records<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_map_records<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t launch_radius_mask(const int *center, const float *radius, int nslots, const Geom &g, unsigned *mask,
                               long long xwords, cudaStream_t st) {
    if (nslots <= 0) return cudaSuccess;
    k_radius_mask<<<(unsigned)nslots, 256, 0, st>>>(center, radius, g, mask, xwords);
    return cudaGetLastError();
}

// Several training images: one thread per slot merges every TI's K best
// and draws (see MultiDrawArgs).  The merge is the reference's std::sort of
// the TIs x K candidates by score (quantileSamplingModule.hpp:101-104),
// which for at most 16 candidates is libstdc++'s insertion sort: stable.
__global__ void k_multi_draw(MultiDrawArgs A) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= A.nslots) return;
    const Slot s = A.slots[b];
    const int nvar = A.nvar;
    unsigned ti = 0, tcell = 0;
    if (s.flags & SLOT_SKIP) {
        // marginal: the TIs' cells end to end (simulation.hpp:586-610)
        unsigned cumulated = 0;
        for (int t = 0; t < A.nti; ++t) cumulated += (unsigned)A.ti_cells[t] * (unsigned)nvar;
        const unsigned position =
            (unsigned)(int)floorf(__fmul_rn(s.seed, __uint2float_rn(cumulated / (unsigned)nvar)));
        cumulated = 0;
        for (int t = 0; t < A.nti; ++t) {
            const unsigned size = (unsigned)A.ti_cells[t] * (unsigned)nvar;
            if (position * (unsigned)nvar < cumulated + size) {
                ti = (unsigned)t;
                tcell = position - cumulated / (unsigned)nvar;
                break;
            }
            cumulated += size;
        }
    } else {
        // delta = sum over continuous variables, then neighbours, of
        // -1 * (w * v * v) in the reference's float order
        // (quantileSamplingModule.hpp:412-457)
        float delta = 0.f;
        const int cnt = A.nb_count[s.node];
        for (int i = 0; i < nvar; ++i) {
            if (A.types[i] != 0) continue;
            for (int j = 0; j < cnt; ++j) {
                const unsigned c = A.nb_cell[(long long)s.node * A.n + j];
                const float v = A.state[(long long)c * nvar + i];
                if (isnan(v)) continue;
                const float w = A.wtab[(long long)A.nb_tpl[(long long)s.node * A.n + j] * nvar + i];
                delta = __fadd_rn(delta, __fmul_rn(-1.f, __fmul_rn(__fmul_rn(w, v), v)));
            }
        }
        const int req = A.ii ? (int)A.ii[s.cell] : -1;
        float v[16];
        int o[16];
        const int m = A.nti * A.K;
        for (int q = 0; q < m; ++q) {
            const int t = q / A.K;
            v[q] = (req < 0 || t == req) ? __fadd_rn(A.vals[t * A.ti_stride + (long long)b * A.K + q % A.K], delta)
                                         : -CUDART_INF_F;
            o[q] = q;
        }
        for (int q = 1; q < m; ++q) {
            const float x = v[q];
            const int y = o[q];
            int j = q;
            while (j > 0 && x > v[j - 1]) {
                v[j] = v[j - 1];
                o[j] = o[j - 1];
                --j;
            }
            v[j] = x;
            o[j] = y;
        }
        const int q = o[s.sel < m ? s.sel : m - 1];
        ti = (unsigned)(q / A.K);
        tcell = A.cells[ti * A.ti_stride + (long long)b * A.K + q % A.K];
    }
    if (A.node_cell) A.node_cell[s.node] = tcell;
    if (A.state) {
        for (int v2 = 0; v2 < nvar; ++v2) {
            float *dst = A.state + (long long)s.cell * nvar + v2;
            if (isnan(*dst)) *dst = A.ti[ti][(long long)tcell * nvar + v2];
        }
    }
    if (A.id_image) A.id_image[s.cell] = tcell * (unsigned)A.nti + ti;
}

cudaError_t launch_multi_draw(const MultiDrawArgs &a, cudaStream_t st) {
    if (a.nslots <= 0) return cudaSuccess;
    if (a.nti < 1 || a.nti > QSK_MAX_TIS || a.nti * a.K > 16) return cudaErrorInvalidValue;
    k_multi_draw<<<(unsigned)((a.nslots + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_mt_prep(const SimPrepArgs &a, unsigned *state, int *pre, cudaStream_t st) {
    k_mt_prep<<<(unsigned)((a.nslots + RP_WARPS - 1) / RP_WARPS), 32 * RP_WARPS, 0, st>>>(a, state, pre);
    return cudaGetLastError();
}

template <int T>
static void launch_replay_team(const ReplayArgs &a, size_t smem, cudaStream_t st) {
    const unsigned blocks = (unsigned)a.nslots;
    if (a.K <= 1) k_replay<1, T><<<blocks, 32 * T, smem, st>>>(a);
    else if (a.K <= 2) k_replay<2, T><<<blocks, 32 * T, smem, st>>>(a);
    else if (a.K <= 4) k_replay<4, T><<<blocks, 32 * T, smem, st>>>(a);
    else if (a.K <= 8) k_replay<8, T><<<blocks, 32 * T, smem, st>>>(a);
    else k_replay<16, T><<<blocks, 32 * T, smem, st>>>(a);
}

cudaError_t launch_hash_select(const ReplayArgs &a, cudaStream_t st) {
    if (a.nslots <= 0) return cudaSuccess;
    if (a.K <= 2) k_hash_select<2><<<(unsigned)a.nslots, HS_THREADS, 0, st>>>(a);
    else if (a.K <= 4) k_hash_select<4><<<(unsigned)a.nslots, HS_THREADS, 0, st>>>(a);
    else if (a.K <= 8) k_hash_select<8><<<(unsigned)a.nslots, HS_THREADS, 0, st>>>(a);
    else k_hash_select<16><<<(unsigned)a.nslots, HS_THREADS, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_replay(const ReplayArgs &a, cudaStream_t st) {
    // One CTA per slot: a team of warps (warp 0 replays, the others help
    // with the generator blocks and the tie super-runs) around one shared
    // state of ~25 KB.  Teams of eight while every slot of the batch gets an
    // SM slot at once (registers allow 4 such CTAs per SM); larger batches
    // take teams of four, 8 CTAs per SM, so that they still run in one wave
    // up to 1184 slots.  A warp per slot with a state of its own (8 warps per
    // SM) measured slower at every batch size of the simulations.
    static std::atomic<int> wave8[64][5];   // per device and K class; 0 until measured (jobs may run in threads)
    const size_t smem = sizeof(WarpShared);
    if (a.nslots <= 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    const int kc = a.K <= 1 ? 0 : a.K <= 2 ? 1 : a.K <= 4 ? 2 : a.K <= 8 ? 3 : 4;
    int wave = wave8[dev][kc].load(std::memory_order_relaxed);
    if (wave == 0) {
        int sms = 0, per_sm = 0;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        const void *fn = kc == 0   ? (const void *)k_replay<1, TEAM_MAX>
                         : kc == 1 ? (const void *)k_replay<2, TEAM_MAX>
                         : kc == 2 ? (const void *)k_replay<4, TEAM_MAX>
                         : kc == 3 ? (const void *)k_replay<8, TEAM_MAX>
                                   : (const void *)k_replay<16, TEAM_MAX>;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * TEAM_MAX, smem)) != cudaSuccess)
            return e;
        wave = sms * (per_sm > 0 ? per_sm : 1);
        wave8[dev][kc].store(wave, std::memory_order_relaxed);
    }
    if (a.nslots <= wave) launch_replay_team<TEAM_MAX>(a, smem, st);
    else launch_replay_team<TEAM_MAX / 2>(a, smem, st);
    return cudaGetLastError();
}

}  // namespace qsk

// Node rows of the tensor-core form: the A operand of a dependency level's
// GEMM (each node's weights and values over the template prefix, in BF16 or
// FP8 E4M3 with a per-node power-of-two scale), the node's validity box, bias
// and tie seed.  Shared by k_tc_nodes (qsk_tc.cu) and the fused level kernel
// k_prep_tc_nodes (qsk_kernels.cu).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp8.h>

#include "qsk_internal.h"

namespace qsk {
namespace {

__device__ __forceinline__ void store_elem(void *base, long long idx, float v, int fmt) {
    if (fmt == 0) {
        reinterpret_cast<__nv_bfloat16 *>(base)[idx] = __float2bfloat16_rn(v);
    } else {
        reinterpret_cast<__nv_fp8_storage_t *>(base)[idx] = __nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
    }
}

// FP8 E4M3 scale of a row whose largest magnitude is mx: the power of two
// that brings mx to at most 448 (the format's largest finite value), so that
// scaling and unscaling are exact
__device__ __forceinline__ float pow2_scale(float mx) {
    if (!(mx > 0.f)) return 1.f;
    int e;
    frexpf(mx / 448.f, &e);   // mx / 448 = f * 2^e, f in [0.5, 1)
    return ldexpf(1.f, e);
}

// slot `warp` of the level (one warp); warps in [nslots, rows) only zero
// their padding row of A
__device__ __forceinline__ void tc_nodes_warp(const TcNodeArgs &A, const int warp, const int lane) {
    if (A.A) {
        // the warp's row of A starts as zeros (the entries below are sparse);
        // a row is Kp * elem bytes, a multiple of 128
        if (warp >= A.rows) return;
        const long long rb = A.Kp * (A.fmt == 1 ? 1 : 2);
        uint4 *row = reinterpret_cast<uint4 *>(static_cast<unsigned char *>(A.A) + (long long)warp * rb);
        for (long long q = lane; q < rb / 16; q += 32) row[q] = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
    }
    if (warp >= A.nslots) return;
    if (A.node_thr && lane == 0) A.node_thr[warp] = 0u;
    const int i = A.nodes[warp];
    const unsigned cell = A.path[A.begin + i];
    const int cnt = A.nb_count[i];
    const int nd = A.nd;
    int mn[QSK_MAXD] = {0, 0, 0, 0}, mx[QSK_MAXD] = {0, 0, 0, 0};
    float amax = 0.f;
    for (int j = lane; j < cnt; j += 32) {
        const int t = A.nb_tpl[(long long)i * A.n + j];
        const unsigned nc = A.nb_cell[(long long)i * A.n + j];
        for (int d = 0; d < nd; ++d) {
            const int o = A.tpl[t * nd + d];
            mn[d] = min(mn[d], o);
            mx[d] = max(mx[d], o);
        }
        for (int v = 0; v < A.nvar; ++v) {
            const float val = nc == cell ? A.init[(long long)nc * A.nvar + v] : A.state[(long long)nc * A.nvar + v];
            const float w = A.wtab[t * A.nvar + v];
            if (isnan(val) || w == 0.f) continue;
            if (A.types[v] == 0) amax = fmaxf(amax, fmaxf(fabsf(w), fabsf(2.f * __fmul_rn(w, val))));
            else amax = fmaxf(amax, fabsf(w));
        }
    }
#pragma unroll
    for (int d = 0; d < QSK_MAXD; ++d)
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
    for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const float scale = A.fmt == 1 ? pow2_scale(amax) : 1.f;
    const float inv = 1.f / scale;
    float bias = 0.f;
    for (int j = lane; j < cnt && A.A; j += 32) {
        const int t = A.nb_tpl[(long long)i * A.n + j];
        const unsigned nc = A.nb_cell[(long long)i * A.n + j];
        for (int v = 0; v < A.nvar; ++v) {
            const float val = nc == cell ? A.init[(long long)nc * A.nvar + v] : A.state[(long long)nc * A.nvar + v];
            const float w = A.wtab[t * A.nvar + v];
            if (isnan(val) || w == 0.f) continue;
            const long long col = (long long)t * A.L + A.var_layer0[v];
            if (A.types[v] == 0) {
                store_elem(A.A, (long long)warp * A.Kp + col, -w * inv, A.fmt);
                store_elem(A.A, (long long)warp * A.Kp + col + 1, 2.f * __fmul_rn(w, val) * inv, A.fmt);
            } else {
                // C categories, C-1 indicator layers: the last category's
                // match is 1 minus the others' (its weight goes to the bias)
                const int C = A.var_ncat[v];
                int ci = -1;
                for (int c = 0; c < C; ++c)
                    if (A.var_catv[v * QSK_CMAX + c] == val) ci = c;
                if (ci < 0) continue;   // no category of the TI: matches nowhere
                if (ci < C - 1) {
                    store_elem(A.A, (long long)warp * A.Kp + col + ci, w * inv, A.fmt);
                } else {
                    for (int c = 0; c < C - 1; ++c) store_elem(A.A, (long long)warp * A.Kp + col + c, -w * inv, A.fmt);
                    bias += w;
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) bias += __shfl_xor_sync(0xffffffffu, bias, o);
    if (lane == 0) {
        A.node_scale[warp] = scale;
        A.node_bias[warp] = bias;
        for (int d = 0; d < 3; ++d) {
            const bool has = d < nd;
            A.node_box[warp * 6 + 2 * d] = has ? -mn[d] : 0;
            A.node_box[warp * 6 + 2 * d + 1] = has ? A.src[d] - mx[d] : 1;
        }
        A.node_seed[warp] = __float_as_uint(A.seeds[i]) ^ (unsigned(i) * 0x85EBCA6Bu);
    }
}

}  // namespace
}  // namespace qsk

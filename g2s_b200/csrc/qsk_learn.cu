// Learned proposal: a small MLP encoder of neighbourhoods, its training
// (forward, backward and Adam, FP32 on the CUDA cores) and the features it
// reads.  The encoder embeds a node's informed neighbourhood (query head)
// and the neighbourhood of every TI cell (pattern head) into one 64-d space;
// the tensor-core top-W kernel (qsk_tc.cu) then proposes, per node, the TI
// cells whose embeddings have the largest inner product with the node's, and
// the exact map scores that shortlist.
//
// Encoder: E = 64 entries x F features (F = nvar values, mask, dx, dy, dz),
// D0 = 64 F -> 256 -> 256 -> 256 (GELU, tanh form of Hendrycks & Gimpel
// 2016, shared) -> 64 (one linear head per side, not normalised).  Training
// pairs (query neighbourhood, TI cell the exact path drew for it) use the
// symmetric InfoNCE loss over the in-batch negatives (logits = q . p / tau).
//
// Entries form a stencil: the template's first 64 offsets, dilated by a
// scale s in 1..nscales.  A node takes the smallest scale whose stencil
// holds most of its informed neighbours (sparse neighbourhoods early on the
// path take a coarse stencil); the TI is embedded once per scale.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "qsk_internal.h"

namespace qsk {
namespace {

constexpr int GT = 64;       // GEMM tile (rows and columns)
constexpr int GK = 16;       // GEMM K step
constexpr int GTHREADS = 256;

// C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C (+ bias[n]),
// op(X) = X or X^T; row-major with leading dimensions.  64 x 64 tiles, each
// thread 4 x 4 outputs.
__global__ void __launch_bounds__(GTHREADS) k_sgemm(int M, int N, int K, const float *__restrict__ A, int lda, int ta,
                                                    const float *__restrict__ B, int ldb, int tb, float *__restrict__ C,
                                                    int ldc, float alpha, float beta, const float *__restrict__ bias) {
    __shared__ float As[GK][GT + 1];
    __shared__ float Bs[GK][GT + 1];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int row0 = blockIdx.y * GT, col0 = blockIdx.x * GT;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int i = threadIdx.x; i < GK * GT; i += GTHREADS) {
            const int kk = i / GT, mm = i % GT;
            const int r = row0 + mm, k = k0 + kk;
            float av = 0.f;
            if (r < M && k < K) av = ta ? A[(long long)k * lda + r] : A[(long long)r * lda + k];
            As[kk][mm] = av;
            const int c = col0 + mm;
            float bv = 0.f;
            if (c < N && k < K) bv = tb ? B[(long long)c * ldb + k] : B[(long long)k * ldb + c];
            Bs[kk][mm] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = As[kk][ty * 4 + u];
                b[u] = Bs[kk][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = row0 + ty * 4 + u;
        if (r >= M) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int c = col0 + tx * 4 + v;
            if (c >= N) continue;
            float x = alpha * acc[u][v];
            if (beta != 0.f) x += beta * C[(long long)r * ldc + c];
            if (bias) x += bias[c];
            C[(long long)r * ldc + c] = x;
        }
    }
}

__device__ __forceinline__ float gelu(float x) {
    const float c = 0.7978845608028654f;   // sqrt(2 / pi)
    return 0.5f * x * (1.f + tanhf(c * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float c = 0.7978845608028654f;
    const float u = c * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * c * (1.f + 3.f * 0.044715f * x * x);
}

__global__ void k_gelu(long long n, const float *__restrict__ pre, float *__restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = gelu(pre[i]);
}
__global__ void k_gelu_back(long long n, const float *__restrict__ pre, float *__restrict__ d) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) d[i] *= gelu_grad(pre[i]);
}

// column sums (bias gradients): out[c] (+)= sum_r d[r][c]
__global__ void k_colsum(int rows, int cols, const float *__restrict__ d, float *__restrict__ out, int accumulate) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += d[(long long)r * cols + c];
    out[c] = accumulate ? out[c] + s : s;
}

// symmetric InfoNCE on logits L = S / tau (B x B, positives on the diagonal):
// loss = (mean_i CE(row i) + mean_j CE(column j)) / 2; writes dS (the
// gradient with respect to S) and adds the loss to *loss
__global__ void k_infonce(int B, float tau, const float *__restrict__ S, float *__restrict__ dS, float *loss) {
    // one warp per row for the row softmax, then one warp per column
    const int w = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (w >= 2 * B) return;
    const bool col = w >= B;
    const int i = col ? w - B : w;
    auto at = [&](int j) { return col ? S[(long long)j * B + i] : S[(long long)i * B + j]; };
    float mx = -INFINITY;
    for (int j = lane; j < B; j += 32) mx = fmaxf(mx, at(j) / tau);
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float se = 0.f;
    for (int j = lane; j < B; j += 32) se += expf(at(j) / tau - mx);
    for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
    const float lse = mx + logf(se);
    const float scale = 0.5f / (float)B / tau;
    for (int j = lane; j < B; j += 32) {
        const float p = expf(at(j) / tau - lse);
        const float g = (p - (j == i ? 1.f : 0.f)) * scale;
        const long long idx = col ? (long long)j * B + i : (long long)i * B + j;
        atomicAdd(&dS[idx], g);
    }
    if (lane == 0) atomicAdd(loss, 0.5f * (lse - at(i) / tau) / (float)B);
}

__global__ void k_adam(long long n, float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// entry of the stencil a neighbour at template offset tp falls in at scale s
// (-1: outside it; the centre is no entry)
__device__ __forceinline__ int stencil_entry(const FeatArgs &A, const int *tp, int s) {
    int idx = 0, st = 1;
    for (int d = 0; d < A.nd; ++d) {
        const int o = tp[d];
        const int a = o < 0 ? -o : o;
        int q = (2 * a + s) / (2 * s);
        if (o < 0) q = -q;
        const int c = q - A.cube_lo[d];
        if (c < 0 || c >= A.cube_dim[d]) return -1;
        idx += c * st;
        st *= A.cube_dim[d];
    }
    return A.cube[idx];
}

// encoder input of nodes: entry e of the row's stencil holds
// [mean of the values of the neighbours falling in it, 1, dx, dy, dz], or
// [0, 0, dx, dy, dz] when none does (the centre and neighbours beyond the
// stencil are not represented; the exact map still uses them); dx, dy, dz
// is the entry's offset (scale included) times inv_radius
__global__ void k_feat_nodes(FeatArgs A) {
    const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (r >= A.rows) return;   // r is the same for the whole warp
    const int i = A.nodes[r];
    const unsigned cell = A.path[A.begin + i];
    const int cnt = A.nb_count[i];
    const int F = A.nvar + 4;
    const int E = min(A.entries, QSK_ENC_ENTRIES);
    const int s = A.row_scale ? A.row_scale[r] : A.scale;
    float *out = A.out + (long long)r * QSK_ENC_ENTRIES * F;
    for (int e = lane; e < QSK_ENC_ENTRIES; e += 32) {
        float *o = out + e * F;
        for (int v = 0; v <= A.nvar; ++v) o[v] = 0.f;
        const int t = e + 1;
        for (int d = 0; d < 3; ++d)
            o[A.nvar + 1 + d] =
                (d < A.nd && t < A.ntpl && e < E) ? float(s * A.tpl[t * A.nd + d]) * A.inv_radius : 0.f;
    }
    // neighbours in their order; the lane owning an entry (e mod 32) adds
    // them up, so every entry's sum has a fixed order
    for (int j0 = 0; j0 < cnt; j0 += 32) {
        const int j = j0 + lane;
        int ent = -1;
        unsigned nc = 0;
        if (j < cnt) {
            const int t = A.nb_tpl[(long long)i * A.n + j];
            nc = A.nb_cell[(long long)i * A.n + j];
            if (t >= 1 && t < A.ntpl && nc != cell) {
                ent = stencil_entry(A, A.tpl + t * A.nd, s);
                if (ent >= E) ent = -1;
            }
        }
        const int m = min(32, cnt - j0);
        for (int jj = 0; jj < m; ++jj) {
            const int e = __shfl_sync(0xffffffffu, ent, jj);
            const unsigned c = __shfl_sync(0xffffffffu, nc, jj);
            if (e >= 0 && (e & 31) == lane) {
                float *o = out + e * F;
                for (int v = 0; v < A.nvar; ++v) {
                    const float x = A.state[(long long)c * A.nvar + v];
                    o[v] += isnan(x) ? 0.f : x;
                }
                o[A.nvar] += 1.f;
            }
        }
    }
    for (int e = lane; e < QSK_ENC_ENTRIES; e += 32) {
        float *o = out + e * F;
        const float c = o[A.nvar];
        if (c > 1.f)
            for (int v = 0; v < A.nvar; ++v) o[v] = o[v] / c;
        o[A.nvar] = c > 0.f ? 1.f : 0.f;
    }
}

// encoder input of TI cells: the stencil's entries around the cell at the
// row's scale (the neighbours a node with a complete neighbourhood has,
// centre excluded)
__global__ void k_feat_cells(FeatArgs A) {
    const long long r = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (r >= A.rows) return;
    const long long p = A.cell_list ? (long long)A.cell_list[r] : A.cell0 + r;
    const int F = A.nvar + 4;
    const int s = A.row_scale ? A.row_scale[r] : A.scale;
    int pc[3] = {0, 0, 0};
    long long rem = p;
    for (int d = 0; d < A.nd; ++d) {
        pc[d] = int(rem % A.src[d]);
        rem /= A.src[d];
    }
    float *out = A.out + r * 64 * F;
    for (int e = lane; e < 64; e += 32) {
        const int t = e + 1;
        float *o = out + e * F;
        long long q = 0, st = 1;
        bool in = p < A.cells && t < A.ntpl && e < A.entries;
        for (int d = 0; d < A.nd; ++d) {
            const int off = t < A.ntpl ? s * A.tpl[t * A.nd + d] : 0;
            const int c = pc[d] + off;
            in &= c >= 0 && c < A.src[d];
            q += (long long)c * st;
            st *= A.src[d];
        }
        for (int v = 0; v < A.nvar; ++v) {
            const float x = in ? A.ti[q * A.nvar + v] : 0.f;
            o[v] = isnan(x) ? 0.f : x;
        }
        o[A.nvar] = in ? 1.f : 0.f;
        for (int d = 0; d < 3; ++d)
            o[A.nvar + 1 + d] =
                (d < A.nd && t < A.ntpl && e < A.entries) ? float(s * A.tpl[t * A.nd + d]) * A.inv_radius : 0.f;
    }
}

// the scale of each node's stencil: the smallest scale whose entries hold at
// least cov_min of its neighbours, else the one holding the most
__global__ void k_node_scale(FeatArgs A) {
    const int r = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (r >= A.rows) return;   // r is the same for the whole warp
    const int i = A.nodes[r];
    const unsigned cell = A.path[A.begin + i];
    const int cnt = A.nb_count[i];
    const int E = min(A.entries, QSK_ENC_ENTRIES);
    int best = 1, bestc = -1;
    for (int s = 1; s <= A.nscales; ++s) {
        int c = 0;
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            const int j = j0 + lane;
            bool in = false;
            if (j < cnt) {
                const int t = A.nb_tpl[(long long)i * A.n + j];
                const unsigned nc = A.nb_cell[(long long)i * A.n + j];
                if (t >= 1 && t < A.ntpl && nc != cell) {
                    const int e = stencil_entry(A, A.tpl + t * A.nd, s);
                    in = e >= 0 && e < E;
                }
            }
            c += __popc(__ballot_sync(0xffffffffu, in));
        }
        if (float(c) >= A.cov_min * float(cnt)) {
            best = s;
            break;
        }
        if (c > bestc) {
            best = s;
            bestc = c;
        }
    }
    if (lane == 0) A.scale_out[r] = best;
}

__global__ void k_to_bf16(long long n, const float *__restrict__ x, uint16_t *__restrict__ y) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const unsigned u = __float_as_uint(x[i]);
        // round to nearest even on the upper 16 bits (finite inputs)
        const unsigned r = u + 0x7FFFu + ((u >> 16) & 1u);
        y[i] = (uint16_t)(r >> 16);
    }
}

// rows idx[0..n) of src (each `cols` floats) into dst, in order
__global__ void k_gather_rows(int n, int cols, const int *__restrict__ idx, const float *__restrict__ src,
                              float *__restrict__ dst) {
    const int r = blockIdx.x;
    if (r >= n) return;
    const float *s = src + (long long)idx[r] * cols;
    float *d = dst + (long long)r * cols;
    for (int c = threadIdx.x; c < cols; c += blockDim.x) d[c] = s[c];
}

// BF16 operand of the tensor-core GEMM: dst (rows_pad x kpad) element
// (r, c) = src[r * ld + c] (tr 0) or src[c * ld + r] (tr 1) for r < rows and
// c < cols, zero elsewhere; 32 x 32 tiles through shared memory, so that
// reads and writes are coalesced either way
__global__ void k_pack_bf16(int rows, int cols, const float *__restrict__ src, long long ld, int tr, int kpad,
                            __nv_bfloat16 *__restrict__ dst) {
    __shared__ float t[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int i = ty; i < 32; i += 8) {
        if (!tr) {
            const int r = r0 + i, c = c0 + tx;
            t[i][tx] = (r < rows && c < cols) ? src[(long long)r * ld + c] : 0.f;
        } else {
            const int c = c0 + i, r = r0 + tx;
            t[tx][i] = (r < rows && c < cols) ? src[(long long)c * ld + r] : 0.f;
        }
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) dst[(long long)(r0 + i) * kpad + c0 + tx] = __float2bfloat16_rn(t[i][tx]);
}

unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_sgemm(int M, int N, int K, const float *A, int lda, int ta, const float *B, int ldb, int tb, float *C,
                         int ldc, float alpha, float beta, const float *bias, cudaStream_t st) {
    if (M <= 0 || N <= 0) return cudaSuccess;
    dim3 grid((unsigned)((N + GT - 1) / GT), (unsigned)((M + GT - 1) / GT));
    k_sgemm<<<grid, GTHREADS, 0, st>>>(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, alpha, beta, bias);
    return cudaGetLastError();
}
cudaError_t launch_gelu(long long n, const float *pre, float *out, cudaStream_t st) {
    k_gelu<<<blocks_for(n, 256), 256, 0, st>>>(n, pre, out);
    return cudaGetLastError();
}
cudaError_t launch_gelu_back(long long n, const float *pre, float *d, cudaStream_t st) {
    k_gelu_back<<<blocks_for(n, 256), 256, 0, st>>>(n, pre, d);
    return cudaGetLastError();
}
cudaError_t launch_colsum(int rows, int cols, const float *d, float *out, int accumulate, cudaStream_t st) {
    k_colsum<<<blocks_for(cols, 128), 128, 0, st>>>(rows, cols, d, out, accumulate);
    return cudaGetLastError();
}
cudaError_t launch_infonce(int B, float tau, const float *S, float *dS, float *loss, cudaStream_t st) {
    k_infonce<<<blocks_for((long long)2 * B * 32, 256), 256, 0, st>>>(B, tau, S, dS, loss);
    return cudaGetLastError();
}
cudaError_t launch_adam(long long n, float *w, const float *g, float *m, float *v, float lr, int t, cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
    k_adam<<<blocks_for(n, 256), 256, 0, st>>>(n, w, g, m, v, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError();
}
cudaError_t launch_pack_bf16(int rows, int cols, const float *src, long long ld, int tr, long long rows_pad, int kpad,
                             void *dst, cudaStream_t st) {
    if (rows_pad <= 0 || kpad <= 0) return cudaSuccess;
    if (rows_pad % 32 || kpad % 32 || rows > rows_pad || cols > kpad) return cudaErrorInvalidValue;
    dim3 grid((unsigned)(kpad / 32), (unsigned)(rows_pad / 32));
    k_pack_bf16<<<grid, dim3(32, 8), 0, st>>>(rows, cols, src, ld, tr, kpad, reinterpret_cast<__nv_bfloat16 *>(dst));
    return cudaGetLastError();
}
cudaError_t launch_feat_nodes(const FeatArgs &a, cudaStream_t st) {
    if (a.rows <= 0) return cudaSuccess;
    k_feat_nodes<<<blocks_for(a.rows * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_feat_cells(const FeatArgs &a, cudaStream_t st) {
    if (a.rows <= 0) return cudaSuccess;
    k_feat_cells<<<blocks_for(a.rows * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_node_scale(const FeatArgs &a, cudaStream_t st) {
    if (a.rows <= 0) return cudaSuccess;
    if (!a.cube || !a.scale_out || a.nscales < 1) return cudaErrorInvalidValue;
    k_node_scale<<<blocks_for(a.rows * 32, 256), 256, 0, st>>>(a);
    return cudaGetLastError();
}
cudaError_t launch_gather_rows(int n, int cols, const int *idx, const float *src, float *dst, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_gather_rows<<<(unsigned)n, 128, 0, st>>>(n, cols, idx, src, dst);
    return cudaGetLastError();
}
cudaError_t launch_to_bf16(long long n, const float *x, uint16_t *y, cudaStream_t st) {
    k_to_bf16<<<blocks_for(n, 256), 256, 0, st>>>(n, x, y);
    return cudaGetLastError();
}

}  // namespace qsk

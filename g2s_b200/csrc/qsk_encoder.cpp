// Host side of the learned proposal's encoder: parameters, Adam state, the
// forward and backward passes over a batch, training on device-resident
// (query, positive) feature pairs, and embedding of feature rows.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/g2s_b200.h"
#include "qsk_host_util.h"
#include "qsk_internal.h"
#include "qsk_encoder.h"

using namespace qsk;

// return a failing status code of a call
#define QSK_RC(expr)                \
    do {                            \
        const int rc_ = (expr);     \
        if (rc_ != QSK_OK) return rc_; \
    } while (0)

namespace qsk {

// parameter layout: W1 [H x D0], b1 [H], W2 [H x H], b2, W3 [H x H], b3
// (the shared trunk), W4q [E x H], b4q [E] (query head), W4p [E x H], b4p
// (TI-pattern head); weights row-major, out x in
void enc_layout(int D0, long long off[ENC_NP + 1], long long &total) {
    const long long sz[ENC_NP] = {(long long)ENC_H * D0, ENC_H, (long long)ENC_H * ENC_H, ENC_H,
                                  (long long)ENC_H * ENC_H, ENC_H, (long long)ENC_E * ENC_H, ENC_E,
                                  (long long)ENC_E * ENC_H, ENC_E};
    total = 0;
    for (int i = 0; i < ENC_NP; ++i) {
        off[i] = total;
        total += sz[i];
    }
    off[ENC_NP] = total;
}

int enc_scratch(qsk_encoder *e, long long rows) {
    if (rows <= e->cap) return QSK_OK;
    const size_t r = size_t(rows);
    QSK_CK(e->h1p.alloc(r * ENC_H));
    QSK_CK(e->h1.alloc(r * ENC_H));
    QSK_CK(e->h2p.alloc(r * ENC_H));
    QSK_CK(e->h2.alloc(r * ENC_H));
    QSK_CK(e->h3p.alloc(r * ENC_H));
    QSK_CK(e->h3.alloc(r * ENC_H));
    QSK_CK(e->y.alloc(r * ENC_E));
    QSK_CK(e->d1.alloc(r * ENC_H));
    QSK_CK(e->d2.alloc(r * ENC_H));
    QSK_CK(e->dz.alloc(r * ENC_E));
    e->cap = rows;
    return QSK_OK;
}

// C = op(A) op(B) (+ bias[n]), op(A) M x K and op(B) K x N as in
// launch_sgemm (ta: A stored K x M; tb: B stored N x K): on the tensor cores
// (op(A) and op(B)^T packed to zero-padded BF16, FP32 accumulation) or in
// FP32 on the CUDA cores
int enc_gemm(qsk_encoder *e, int M, int N, int K, const float *A, int lda, int ta, const float *B, int ldb, int tb,
             float *C, int ldc, const float *bias, cudaStream_t st) {
    if (!e->tensor) {
        QSK_CK(launch_sgemm(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, 1.f, 0.f, bias, st));
        return QSK_OK;
    }
    if (M <= 0 || N <= 0) return QSK_OK;
    const int kpad = (K + 63) / 64 * 64;
    const long long ar = (M + 127LL) / 128 * 128;
    const int bn = tc_gemm_bn(N);
    const long long br = (N + bn - 1LL) / bn * bn;
    QSK_CK(e->pa.ensure(size_t(ar) * kpad));
    QSK_CK(e->pb.ensure(size_t(br) * kpad));
    QSK_CK(launch_pack_bf16(M, K, A, lda, ta, ar, kpad, e->pa.p, st));
    QSK_CK(launch_pack_bf16(N, K, B, ldb, tb ? 0 : 1, br, kpad, e->pb.p, st));
    TcGemmArgs g;
    g.M = M;
    g.N = N;
    g.kpad = kpad;
    g.C = C;
    g.ldc = ldc;
    g.bias = bias;
    g.status = e->status.p;
    QSK_CK(launch_tc_gemm(e->pa.p, ar, e->pb.p, br, g, st));
    return QSK_OK;
}

int enc_check(qsk_encoder *e, cudaStream_t st) {
    int v = 0;
    QSK_CK(cudaMemcpyAsync(&v, e->status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    QSK_CK(cudaStreamSynchronize(st));
    if (v != 0) {
        QSK_CK(cudaMemsetAsync(e->status.p, 0, sizeof(int), st));
        return set_error(QSK_ERR_DEVICE, "encoder: a tensor-core product's pipeline wait ran out (status %d)", v);
    }
    return QSK_OK;
}

// rows x D0 inputs x -> embeddings e->y (rows x E) by the trunk and a head:
// rows [0, nq) the query head, rows [nq, rows) the TI-pattern head;
// activations kept for the backward pass
int enc_forward(qsk_encoder *e, long long rows, long long nq, const float *x, cudaStream_t st) {
    int rc = enc_scratch(e, rows);
    if (rc) return rc;
    const float *w = e->w.p;
    const long long *o = e->off;
    const int R = int(rows), Q = int(nq);
    QSK_RC(enc_gemm(e, R, ENC_H, e->D0, x, e->D0, 0, w + o[0], e->D0, 1, e->h1p.p, ENC_H, w + o[1], st));
    QSK_CK(launch_gelu((long long)R * ENC_H, e->h1p.p, e->h1.p, st));
    QSK_RC(enc_gemm(e, R, ENC_H, ENC_H, e->h1.p, ENC_H, 0, w + o[2], ENC_H, 1, e->h2p.p, ENC_H, w + o[3], st));
    QSK_CK(launch_gelu((long long)R * ENC_H, e->h2p.p, e->h2.p, st));
    QSK_RC(enc_gemm(e, R, ENC_H, ENC_H, e->h2.p, ENC_H, 0, w + o[4], ENC_H, 1, e->h3p.p, ENC_H, w + o[5], st));
    QSK_CK(launch_gelu((long long)R * ENC_H, e->h3p.p, e->h3.p, st));
    if (Q > 0)
        QSK_RC(enc_gemm(e, Q, ENC_E, ENC_H, e->h3.p, ENC_H, 0, w + o[6], ENC_H, 1, e->y.p, ENC_E, w + o[7], st));
    if (R > Q)
        QSK_RC(enc_gemm(e, R - Q, ENC_E, ENC_H, e->h3.p + size_t(Q) * ENC_H, ENC_H, 0, w + o[8], ENC_H, 1,
                        e->y.p + size_t(Q) * ENC_E, ENC_E, w + o[9], st));
    return QSK_OK;
}

// gradient of the parameters from dL/dy (e->dz on entry, rows x E), after
// enc_forward on the same rows (the first nq by the query head); gradients
// overwritten in e->g
int enc_backward(qsk_encoder *e, long long rows, long long nq, const float *x) {
    const float *w = e->w.p;
    float *g = e->g.p;
    const long long *o = e->off;
    const int R = int(rows), Q = int(nq);
    cudaStream_t st = e->st;
    // heads: dW4 = dz^T h3, db4 = colsum dz, dh3 = dz W4 (per head's rows)
    QSK_CK(cudaMemsetAsync(g + o[6], 0, sizeof(float) * size_t(o[10] - o[6]), st));
    if (Q > 0) {
        QSK_RC(enc_gemm(e, ENC_E, ENC_H, Q, e->dz.p, ENC_E, 1, e->h3.p, ENC_H, 0, g + o[6], ENC_H, nullptr, st));
        QSK_CK(launch_colsum(Q, ENC_E, e->dz.p, g + o[7], 0, st));
        QSK_RC(enc_gemm(e, Q, ENC_H, ENC_E, e->dz.p, ENC_E, 0, w + o[6], ENC_H, 0, e->d1.p, ENC_H, nullptr, st));
    }
    if (R > Q) {
        const float *dzp = e->dz.p + size_t(Q) * ENC_E;
        QSK_RC(enc_gemm(e, ENC_E, ENC_H, R - Q, dzp, ENC_E, 1, e->h3.p + size_t(Q) * ENC_H, ENC_H, 0, g + o[8], ENC_H,
                        nullptr, st));
        QSK_CK(launch_colsum(R - Q, ENC_E, dzp, g + o[9], 0, st));
        QSK_RC(enc_gemm(e, R - Q, ENC_H, ENC_E, dzp, ENC_E, 0, w + o[8], ENC_H, 0, e->d1.p + size_t(Q) * ENC_H, ENC_H,
                        nullptr, st));
    }
    QSK_CK(launch_gelu_back((long long)R * ENC_H, e->h3p.p, e->d1.p, st));
    // layer 3
    QSK_RC(enc_gemm(e, ENC_H, ENC_H, R, e->d1.p, ENC_H, 1, e->h2.p, ENC_H, 0, g + o[4], ENC_H, nullptr, st));
    QSK_CK(launch_colsum(R, ENC_H, e->d1.p, g + o[5], 0, st));
    QSK_RC(enc_gemm(e, R, ENC_H, ENC_H, e->d1.p, ENC_H, 0, w + o[4], ENC_H, 0, e->d2.p, ENC_H, nullptr, st));
    QSK_CK(launch_gelu_back((long long)R * ENC_H, e->h2p.p, e->d2.p, st));
    // layer 2
    QSK_RC(enc_gemm(e, ENC_H, ENC_H, R, e->d2.p, ENC_H, 1, e->h1.p, ENC_H, 0, g + o[2], ENC_H, nullptr, st));
    QSK_CK(launch_colsum(R, ENC_H, e->d2.p, g + o[3], 0, st));
    QSK_RC(enc_gemm(e, R, ENC_H, ENC_H, e->d2.p, ENC_H, 0, w + o[2], ENC_H, 0, e->d1.p, ENC_H, nullptr, st));
    QSK_CK(launch_gelu_back((long long)R * ENC_H, e->h1p.p, e->d1.p, st));
    // layer 1 (the input needs no gradient)
    QSK_RC(enc_gemm(e, ENC_H, e->D0, R, e->d1.p, ENC_H, 1, x, e->D0, 0, g + o[0], e->D0, nullptr, st));
    QSK_CK(launch_colsum(R, ENC_H, e->d1.p, g + o[1], 0, st));
    return QSK_OK;
}

// loss and parameter gradients of one batch of B pairs stacked as 2B input
// rows (queries first, positives after) in e->xb
int enc_loss_grad(qsk_encoder *e, int B, float tau) {
    int rc = enc_forward(e, 2LL * B, B, e->xb.p, e->st);
    if (rc) return rc;
    QSK_CK(e->S.ensure(size_t(B) * B));
    QSK_CK(e->dS.ensure(size_t(B) * B));
    QSK_CK(e->loss.ensure(1));
    const float *Q = e->y.p, *P = e->y.p + (size_t)B * ENC_E;
    cudaStream_t st = e->st;
    // the logits and their gradient stay FP32 in either mode: the column
    // sums of dS nearly cancel (every softmax row and column sums to one), so
    // the heads' bias gradients are small differences that BF16 operands
    // would swamp; these B x B x 64 products are a small part of a step
    // S = Q P^T
    QSK_CK(launch_sgemm(B, B, ENC_E, Q, ENC_E, 0, P, ENC_E, 1, e->S.p, B, 1.f, 0.f, nullptr, st));
    QSK_CK(cudaMemsetAsync(e->dS.p, 0, sizeof(float) * size_t(B) * B, st));
    QSK_CK(cudaMemsetAsync(e->loss.p, 0, sizeof(float), st));
    QSK_CK(launch_infonce(B, tau, e->S.p, e->dS.p, e->loss.p, st));
    // dQ = dS P, dP = dS^T Q
    float *dQ = e->dz.p, *dP = e->dz.p + (size_t)B * ENC_E;
    QSK_CK(launch_sgemm(B, ENC_E, B, e->dS.p, B, 0, P, ENC_E, 0, dQ, ENC_E, 1.f, 0.f, nullptr, st));
    QSK_CK(launch_sgemm(B, ENC_E, B, e->dS.p, B, 1, Q, ENC_E, 0, dP, ENC_E, 1.f, 0.f, nullptr, st));
    return enc_backward(e, 2LL * B, B, e->xb.p);
}

}  // namespace qsk

extern "C" {

int qsk_encoder_create(int device, int nvar, unsigned seed, qsk_encoder **out) {
    if (!out || nvar < 1 || nvar > 8) return set_error(QSK_ERR_ARG, "encoder: nvar %d (1..8)", nvar);
    DeviceGuard dg(device);
    auto *e = new qsk_encoder();
    e->device = device;
    e->nvar = nvar;
    e->F = nvar + 4;
    e->D0 = QSK_ENC_ENTRIES * e->F;
    enc_layout(e->D0, e->off, e->nparam);
    cudaError_t ce = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        delete e;
        return set_error(QSK_ERR_CUDA, "encoder stream: %s", cudaGetErrorString(ce));
    }
    // uniform (-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases, from mt19937(seed)
    std::vector<float> w(size_t(e->nparam), 0.f);
    std::mt19937 rng(seed);
    const int fan[5] = {e->D0, ENC_H, ENC_H, ENC_H, ENC_H};
    for (int l = 0; l < 5; ++l) {
        const float a = 1.f / std::sqrt(float(fan[l]));
        std::uniform_real_distribution<float> u(-a, a);
        for (long long i = e->off[2 * l]; i < e->off[2 * l + 1]; ++i) w[size_t(i)] = u(rng);
    }
    int rc = QSK_OK;
    if (e->status.alloc(1) != cudaSuccess || cudaMemsetAsync(e->status.p, 0, sizeof(int), e->st) != cudaSuccess ||
        e->w.upload(w.data(), w.size(), e->st) != cudaSuccess || e->g.alloc(w.size()) != cudaSuccess ||
        e->m.alloc(w.size()) != cudaSuccess || e->v.alloc(w.size()) != cudaSuccess ||
        cudaMemsetAsync(e->m.p, 0, sizeof(float) * w.size(), e->st) != cudaSuccess ||
        cudaMemsetAsync(e->v.p, 0, sizeof(float) * w.size(), e->st) != cudaSuccess ||
        cudaStreamSynchronize(e->st) != cudaSuccess)
        rc = set_error(QSK_ERR_NOMEM, "encoder parameters");
    if (rc) {
        qsk_encoder_destroy(e);
        return rc;
    }
    *out = e;
    return QSK_OK;
}

int qsk_encoder_destroy(qsk_encoder *e) {
    if (!e) return QSK_OK;
    {
        DeviceGuard dg(e->device);
        cudaStreamSynchronize(e->st);
        e->w.release();
        e->g.release();
        e->m.release();
        e->v.release();
        e->xq.release();
        e->xp.release();
        e->xb.release();
        if (e->st) cudaStreamDestroy(e->st);
    }
    delete e;
    return QSK_OK;
}

long long qsk_encoder_param_count(const qsk_encoder *e) { return e ? e->nparam : -1; }
int qsk_encoder_input_dim(const qsk_encoder *e) { return e ? e->D0 : -1; }

int qsk_gemm_bf16(int device, int M, int N, int K, const float *A, const float *B, const float *bias, float *C) {
    if (M < 1 || N < 1 || K < 1 || !A || !B || !C) return set_error(QSK_ERR_ARG, "gemm: arguments");
    DeviceGuard dg(device);
    cudaStream_t st = nullptr;
    QSK_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    const int kpad = (K + 63) / 64 * 64, bn = tc_gemm_bn(N);
    const long long ar = (M + 127LL) / 128 * 128, br = (N + bn - 1LL) / bn * bn;
    DBuf<float> a, b, bi, c;
    DBuf<unsigned short> pa, pb;
    DBuf<int> status;
    QSK_CK(a.upload(A, size_t(M) * K, st));
    QSK_CK(b.upload(B, size_t(N) * K, st));
    if (bias) QSK_CK(bi.upload(bias, size_t(N), st));
    QSK_CK(c.alloc(size_t(M) * N));
    QSK_CK(pa.alloc(size_t(ar) * kpad));
    QSK_CK(pb.alloc(size_t(br) * kpad));
    QSK_CK(status.alloc(1));
    QSK_CK(cudaMemsetAsync(status.p, 0, sizeof(int), st));
    QSK_CK(launch_pack_bf16(M, K, a.p, K, 0, ar, kpad, pa.p, st));
    QSK_CK(launch_pack_bf16(N, K, b.p, K, 0, br, kpad, pb.p, st));
    TcGemmArgs g;
    g.M = M;
    g.N = N;
    g.kpad = kpad;
    g.C = c.p;
    g.ldc = N;
    g.bias = bias ? bi.p : nullptr;
    g.status = status.p;
    QSK_CK(launch_tc_gemm(pa.p, ar, pb.p, br, g, st));
    int v = 0;
    QSK_CK(cudaMemcpyAsync(C, c.p, sizeof(float) * size_t(M) * N, cudaMemcpyDeviceToHost, st));
    QSK_CK(cudaMemcpyAsync(&v, status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    QSK_CK(cudaStreamSynchronize(st));
    if (v != 0) return set_error(QSK_ERR_DEVICE, "gemm: a pipeline wait ran out (status %d)", v);
    return QSK_OK;
}

int qsk_encoder_set_tensor_cores(qsk_encoder *e, int on) {
    if (!e) return set_error(QSK_ERR_ARG, "null argument");
    e->tensor = on != 0;
    return QSK_OK;
}

int qsk_encoder_set_scales(qsk_encoder *e, int nscales, float cov_min) {
    if (!e) return set_error(QSK_ERR_ARG, "null argument");
    if (nscales < 1 || nscales > 16 || !(cov_min >= 0.f && cov_min <= 1.f))
        return set_error(QSK_ERR_ARG, "scales %d, coverage %g", nscales, double(cov_min));
    e->nscales = nscales;
    e->cov_min = cov_min;
    return QSK_OK;
}

int qsk_encoder_get_weights(const qsk_encoder *e, float *out) {
    if (!e || !out) return set_error(QSK_ERR_ARG, "null argument");
    DeviceGuard dg(e->device);
    QSK_CK(cudaMemcpyAsync(out, e->w.p, sizeof(float) * size_t(e->nparam), cudaMemcpyDeviceToHost, e->st));
    QSK_CK(cudaStreamSynchronize(e->st));
    return QSK_OK;
}

int qsk_encoder_set_weights(qsk_encoder *e, const float *w) {
    if (!e || !w) return set_error(QSK_ERR_ARG, "null argument");
    DeviceGuard dg(e->device);
    QSK_CK(cudaMemcpyAsync(e->w.p, w, sizeof(float) * size_t(e->nparam), cudaMemcpyHostToDevice, e->st));
    QSK_CK(cudaMemsetAsync(e->m.p, 0, sizeof(float) * size_t(e->nparam), e->st));
    QSK_CK(cudaMemsetAsync(e->v.p, 0, sizeof(float) * size_t(e->nparam), e->st));
    e->t = 0;
    QSK_CK(cudaStreamSynchronize(e->st));
    return QSK_OK;
}

int qsk_encoder_loss_grad(qsk_encoder *e, int B, const float *xq, const float *xp, float tau, float *loss, float *grad) {
    if (!e || B < 1 || !xq || !xp || !loss || !(tau > 0.f)) return set_error(QSK_ERR_ARG, "encoder loss: arguments");
    DeviceGuard dg(e->device);
    const size_t rowf = size_t(e->D0);
    QSK_CK(e->xb.ensure(2 * size_t(B) * rowf));
    QSK_CK(cudaMemcpyAsync(e->xb.p, xq, sizeof(float) * B * rowf, cudaMemcpyHostToDevice, e->st));
    QSK_CK(cudaMemcpyAsync(e->xb.p + size_t(B) * rowf, xp, sizeof(float) * B * rowf, cudaMemcpyHostToDevice, e->st));
    int rc = enc_loss_grad(e, B, tau);
    if (rc) return rc;
    QSK_CK(cudaMemcpyAsync(loss, e->loss.p, sizeof(float), cudaMemcpyDeviceToHost, e->st));
    if (grad) QSK_CK(cudaMemcpyAsync(grad, e->g.p, sizeof(float) * size_t(e->nparam), cudaMemcpyDeviceToHost, e->st));
    return enc_check(e, e->st);
}

int qsk_encoder_embed(qsk_encoder *e, int head, long long rows, const float *x, float *out) {
    if (!e || rows < 1 || !x || !out || (head != 0 && head != 1)) return set_error(QSK_ERR_ARG, "encoder embed: arguments");
    DeviceGuard dg(e->device);
    const size_t rowf = size_t(e->D0);
    const long long chunk = 65536;
    QSK_CK(e->xb.ensure(size_t(std::min(rows, chunk)) * rowf));
    for (long long r0 = 0; r0 < rows; r0 += chunk) {
        const long long n = std::min(chunk, rows - r0);
        QSK_CK(cudaMemcpyAsync(e->xb.p, x + size_t(r0) * rowf, sizeof(float) * size_t(n) * rowf, cudaMemcpyHostToDevice,
                               e->st));
        int rc = enc_forward(e, n, head == 0 ? n : 0, e->xb.p, e->st);
        if (rc) return rc;
        QSK_CK(cudaMemcpyAsync(out + size_t(r0) * ENC_E, e->y.p, sizeof(float) * size_t(n) * ENC_E, cudaMemcpyDeviceToHost,
                               e->st));
    }
    return enc_check(e, e->st);
}

int qsk_encoder_add_pairs_host(qsk_encoder *e, long long n, const float *xq, const float *xp) {
    if (!e || n < 1 || !xq || !xp) return set_error(QSK_ERR_ARG, "encoder pairs: arguments");
    DeviceGuard dg(e->device);
    const size_t rowf = size_t(e->D0);
    if (e->npairs + n > e->pair_cap) {
        const long long cap = std::max<long long>(e->npairs + n, 2 * e->pair_cap);
        DBuf<float> q2, p2;
        QSK_CK(q2.alloc(size_t(cap) * rowf));
        QSK_CK(p2.alloc(size_t(cap) * rowf));
        if (e->npairs) {
            QSK_CK(cudaMemcpyAsync(q2.p, e->xq.p, sizeof(float) * size_t(e->npairs) * rowf, cudaMemcpyDeviceToDevice, e->st));
            QSK_CK(cudaMemcpyAsync(p2.p, e->xp.p, sizeof(float) * size_t(e->npairs) * rowf, cudaMemcpyDeviceToDevice, e->st));
            QSK_CK(cudaStreamSynchronize(e->st));
        }
        e->xq.swap(q2);
        e->xp.swap(p2);
        e->pair_cap = cap;
    }
    QSK_CK(cudaMemcpyAsync(e->xq.p + size_t(e->npairs) * rowf, xq, sizeof(float) * size_t(n) * rowf,
                           cudaMemcpyHostToDevice, e->st));
    QSK_CK(cudaMemcpyAsync(e->xp.p + size_t(e->npairs) * rowf, xp, sizeof(float) * size_t(n) * rowf,
                           cudaMemcpyHostToDevice, e->st));
    QSK_CK(cudaStreamSynchronize(e->st));
    e->npairs += n;
    return QSK_OK;
}

int qsk_encoder_pairs(const qsk_encoder *e, long long *count) {
    if (!e || !count) return set_error(QSK_ERR_ARG, "null argument");
    *count = e->npairs;
    return QSK_OK;
}

int qsk_encoder_get_pairs(const qsk_encoder *e, long long first, long long n, float *xq, float *xp) {
    if (!e || (n > 0 && (!xq || !xp))) return set_error(QSK_ERR_ARG, "null argument");
    if (first < 0 || n < 0 || first + n > e->npairs)
        return set_error(QSK_ERR_ARG, "pairs [%lld, %lld) of %lld", first, first + n, e->npairs);
    if (n == 0) return QSK_OK;
    DeviceGuard dg(e->device);
    const size_t row = size_t(e->D0), at = size_t(first) * row, cnt = size_t(n) * row;
    QSK_CK(cudaMemcpyAsync(xq, e->xq.p + at, sizeof(float) * cnt, cudaMemcpyDeviceToHost, e->st));
    QSK_CK(cudaMemcpyAsync(xp, e->xp.p + at, sizeof(float) * cnt, cudaMemcpyDeviceToHost, e->st));
    QSK_CK(cudaStreamSynchronize(e->st));
    return QSK_OK;
}

int qsk_encoder_clear_pairs(qsk_encoder *e) {
    if (!e) return set_error(QSK_ERR_ARG, "null argument");
    e->npairs = 0;
    return QSK_OK;
}

int qsk_encoder_train(qsk_encoder *e, int epochs, int batch, float lr, float tau, unsigned seed, float *last_loss) {
    if (!e || epochs < 1 || batch < 2 || !(lr > 0.f) || !(tau > 0.f))
        return set_error(QSK_ERR_ARG, "encoder train: arguments");
    if (e->npairs < batch) return set_error(QSK_ERR_ARG, "encoder train: %lld pairs for a batch of %d", e->npairs, batch);
    DeviceGuard dg(e->device);
    const size_t rowf = size_t(e->D0);
    QSK_CK(e->xb.ensure(2 * size_t(batch) * rowf));
    std::mt19937 rng(seed);
    std::vector<int> perm(size_t(e->npairs));
    DBuf<int> dperm;
    QSK_CK(dperm.alloc(perm.size()));
    float l = 0.f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (size_t i = 0; i < perm.size(); ++i) perm[i] = int(i);
        std::shuffle(perm.begin(), perm.end(), rng);
        QSK_CK(cudaMemcpyAsync(dperm.p, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, e->st));
        for (long long b0 = 0; b0 + batch <= e->npairs; b0 += batch) {
            QSK_CK(launch_gather_rows(batch, int(rowf), dperm.p + b0, e->xq.p, e->xb.p, e->st));
            QSK_CK(launch_gather_rows(batch, int(rowf), dperm.p + b0, e->xp.p, e->xb.p + size_t(batch) * rowf, e->st));
            int rc = enc_loss_grad(e, batch, tau);
            if (rc) return rc;
            QSK_CK(launch_adam(e->nparam, e->w.p, e->g.p, e->m.p, e->v.p, lr, ++e->t, e->st));
        }
        QSK_CK(cudaMemcpyAsync(&l, e->loss.p, sizeof(float), cudaMemcpyDeviceToHost, e->st));
        if (int rc = enc_check(e, e->st)) return rc;
    }
    if (last_loss) *last_loss = l;
    return QSK_OK;
}

}  // extern "C"

// The learned proposal's encoder object, shared by the encoder host code
// (qsk_encoder.cpp) and the simulation engine (qsk_host.cpp).
#pragma once

#include <cuda_runtime.h>

#include "qsk_host_util.h"
#include "qsk_internal.h"

namespace qsk {
constexpr int ENC_H = 256;   // hidden width
constexpr int ENC_E = 64;    // embedding width
constexpr int ENC_NP = 10;   // parameter blocks: trunk (3 layers), query head, TI-pattern head
}  // namespace qsk

struct qsk_encoder {
    int device = 0;
    int nvar = 1, F = 5, D0 = 320;
    // stencil scales of the inputs: the TI is embedded at scales 1..nscales;
    // a node takes the smallest holding cov_min of its neighbours
    int nscales = 4;
    float cov_min = 0.9f;
    // matrix products on the tensor cores (BF16 operands, FP32 accumulation)
    // or, when false, on the CUDA cores in FP32
    bool tensor = true;
    qsk::DBuf<unsigned short> pa, pb;   // packed BF16 operands of one product
    qsk::DBuf<int> status;              // DEV_TC_WAIT from the tensor-core kernel
    long long off[qsk::ENC_NP + 1] = {};
    long long nparam = 0;
    cudaStream_t st = nullptr;
    qsk::DBuf<float> w, g, m, v;   // parameters, gradients, Adam moments
    int t = 0;                     // Adam steps taken
    // activations of the last forward pass (rows <= cap)
    long long cap = 0;
    qsk::DBuf<float> h1p, h1, h2p, h2, h3p, h3, y, d1, d2, dz;
    qsk::DBuf<float> xb;           // input rows of a batch / an embedding chunk
    qsk::DBuf<float> S, dS, loss;  // batch similarities and their gradient
    // training pairs (device): query and positive feature rows
    long long npairs = 0, pair_cap = 0;
    qsk::DBuf<float> xq, xp;
};

namespace qsk {
// rows x D0 inputs -> embeddings in e->y (rows x 64), rows [0, nq) by the
// query head and the rest by the TI-pattern head, on stream st
int enc_forward(qsk_encoder *e, long long rows, long long nq, const float *x, cudaStream_t st);
// QSK_OK unless a tensor-core product of the encoder ran out of a wait
// (synchronises st); clears the flag
int enc_check(qsk_encoder *e, cudaStream_t st);
}  // namespace qsk

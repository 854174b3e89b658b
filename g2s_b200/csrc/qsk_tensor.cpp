// Host side of the tensor-core (tcgen05) shortlist: the C ABI entry that
// runs the GEMM-with-shortlist kernel on caller data.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/g2s_b200.h"
#include "qsk_host_util.h"
#include "qsk_internal.h"

using namespace qsk;

namespace {

long long round_up(long long x, long long m) { return (x + m - 1) / m * m; }

}  // namespace

extern "C" {

int qsk_tc_topk(int device, int fmt, int B, long long N, int K, const void *queries, const void *rows,
                const float *q_scale, const float *q_bias, const float *p_scale, const unsigned *q_seed,
                const int *q_box, int X, int Y, int W, int ranges, unsigned long long *out_key, unsigned *out_pos) {
    if (fmt != 0 && fmt != 1) return set_error(QSK_ERR_ARG, "fmt %d (0: BF16, 1: FP8 E4M3)", fmt);
    if (B < 1 || N < 1 || K < 1 || !queries || !rows || !q_box || !out_key || !out_pos)
        return set_error(QSK_ERR_ARG, "empty or null argument");
    if (N > (1LL << 31)) return set_error(QSK_ERR_UNSUPPORTED, "%lld rows (at most 2^31)", N);
    if (!tc_supported_width(W)) return set_error(QSK_ERR_UNSUPPORTED, "shortlist width %d (8, 16 or 32)", W);
    if (ranges < 1 || X < 1 || Y < 1) return set_error(QSK_ERR_ARG, "ranges %d, X %d, Y %d", ranges, X, Y);
    DeviceGuard dg(device);
    const int elem = fmt == 0 ? 2 : 1;
    const long long Kp = round_up(K, 128 / elem);
    const long long Bp = round_up(B, 128), Np = round_up(N, 256);
    cudaStream_t st = nullptr;
    QSK_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    DBuf<unsigned char> dA, dP;
    DBuf<float> dqs, dqb, dps;
    DBuf<unsigned> dseed, dpos;
    DBuf<int> dbox, dstat;
    DBuf<unsigned long long> dkey;
    QSK_CK(dA.alloc(size_t(Bp * Kp * elem)));
    QSK_CK(dP.alloc(size_t(Np * Kp * elem)));
    QSK_CK(cudaMemsetAsync(dA.p, 0, size_t(Bp * Kp * elem), st));
    QSK_CK(cudaMemsetAsync(dP.p, 0, size_t(Np * Kp * elem), st));
    QSK_CK(cudaMemcpy2DAsync(dA.p, size_t(Kp * elem), queries, size_t(K) * elem, size_t(K) * elem, size_t(B),
                             cudaMemcpyHostToDevice, st));
    QSK_CK(cudaMemcpy2DAsync(dP.p, size_t(Kp * elem), rows, size_t(K) * elem, size_t(K) * elem, size_t(N),
                             cudaMemcpyHostToDevice, st));
    if (q_scale) QSK_CK(dqs.upload(q_scale, size_t(B), st));
    if (q_bias) QSK_CK(dqb.upload(q_bias, size_t(B), st));
    if (p_scale) QSK_CK(dps.upload(p_scale, size_t((N + 255) / 256), st));
    if (q_seed) QSK_CK(dseed.upload(q_seed, size_t(B), st));
    QSK_CK(dbox.upload(q_box, size_t(B) * 6, st));
    const size_t nout = size_t(B) * size_t(ranges) * size_t(W);
    QSK_CK(dkey.alloc(nout));
    QSK_CK(dpos.alloc(nout));
    QSK_CK(dstat.alloc(1));
    QSK_CK(cudaMemsetAsync(dstat.p, 0, sizeof(int), st));
    TcArgs a{};
    a.n_nodes = B;
    a.n_pos = N;
    a.n_tiles = Np / 256;
    a.ranges = ranges;
    a.tiles_per_range = int((a.n_tiles + ranges - 1) / ranges);
    a.kblocks = int(Kp * elem / 128);
    a.tile_kblocks = nullptr;
    a.node_scale = q_scale ? dqs.p : nullptr;
    a.node_bias = q_bias ? dqb.p : nullptr;
    a.pos_scale = p_scale ? dps.p : nullptr;
    a.node_seed = q_seed ? dseed.p : nullptr;
    a.node_box = dbox.p;
    a.X = X;
    a.Y = Y;
    a.node_thr = nullptr;   // per-range top W, as documented (no shared bound across ranges)
    a.out_key = dkey.p;
    a.out_pos = dpos.p;
    a.status = dstat.p;
    QSK_CK(launch_tc_shortlist(fmt, W, dA.p, Bp, dP.p, Np, Kp, a, st));
    int status = 0;
    QSK_CK(cudaMemcpyAsync(&status, dstat.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    QSK_CK(cudaMemcpyAsync(out_key, dkey.p, nout * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    QSK_CK(cudaMemcpyAsync(out_pos, dpos.p, nout * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    QSK_CK(cudaStreamSynchronize(st));
    if (status != DEV_OK) return set_error(QSK_ERR_DEVICE, "tensor-core shortlist: device status %d", status);
    return QSK_OK;
}

}  // extern "C"

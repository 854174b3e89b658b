// Peak-rate microbenchmarks of this GPU: the roofline denominators the
// library's kernels are measured against where no driver-measured figure
// exists (FP32 CUDA-core FMA, 32-bit integer logic, tcgen05 BF16 and FP8
// dense MMA).  Each kernel runs long independent chains so that the
// measured rate is the pipe's throughput, not its latency.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/g2s_b200.h"
#include "qsk_host_util.h"
#include "qsk_internal.h"

namespace qsk {
namespace {

constexpr int PK_THREADS = 256;
constexpr int PK_CHAINS = 8;

// 8 independent FMA chains per thread
__global__ void __launch_bounds__(PK_THREADS) k_peak_ffma(float *out, int iters, float a, float b) {
    float x[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) x[c] = float(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < PK_CHAINS; ++c) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s += x[c];
    if (s == 1234.5f) out[threadIdx.x] = s;   // keeps the chains live
}

// 8 independent three-input logic chains per thread (LOP3)
__global__ void __launch_bounds__(PK_THREADS) k_peak_lop3(unsigned *out, int iters, unsigned a, unsigned b) {
    unsigned x[PK_CHAINS];
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) x[c] = threadIdx.x * 2654435761u + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < PK_CHAINS; ++c) asm("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x[c]) : "r"(a), "r"(b));
    }
    unsigned s = 0;
#pragma unroll
    for (int c = 0; c < PK_CHAINS; ++c) s ^= x[c];
    if (s == 0x12345u) out[threadIdx.x] = s;
}

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// One CTA per SM: a single thread issues M=128 x N=256 MMAs back to back on
// operands resident in shared memory (128-byte swizzled K-major tiles of
// zeros), accumulating in TMEM; a commit per 64 MMAs keeps at most one
// batch outstanding.  Every wait is bounded (status on expiry).
template <int KIND>
__global__ void __launch_bounds__(128, 1) k_peak_mma(int iters, int *status) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bar;
    __shared__ unsigned tmem_base;
    // 1024-byte aligned tiles (the swizzle atom): A 128 x 128 B, B 256 x 128 B
    const unsigned raw = smem_addr(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *sa = smem, *sb = smem + 16384;
    for (int i = threadIdx.x; i < (16384 + 32768) / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0, 0, 0, 0);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_addr(&tmem_base))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;
    if (threadIdx.x == 0) {
        auto desc = [](unsigned a) {
            uint64_t d = (uint64_t)((a & 0x3FFFFu) >> 4);
            d |= (uint64_t)1 << 16;
            d |= (uint64_t)(1024 >> 4) << 32;
            d |= (uint64_t)1 << 46;
            d |= (uint64_t)2 << 61;
            return d;
        };
        const uint64_t ad = desc(smem_addr(sa)), bd = desc(smem_addr(sb));
        const unsigned idesc = (1u << 4) | ((KIND == 0 ? 1u : 0u) << 7) | ((KIND == 0 ? 1u : 0u) << 10) |
                               (unsigned(256 >> 3) << 17) | (unsigned(128 >> 4) << 24);
        unsigned phase = 0;
        for (int i = 0; i < iters; ++i) {
#pragma unroll
            for (int k = 0; k < 64; ++k) {
                const uint64_t a2 = ad + (uint64_t)(2 * (k & 3)), b2 = bd + (uint64_t)(2 * (k & 3));
                const unsigned acc = (i | k) != 0;
                if (KIND == 0)
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(a2), "l"(b2), "r"(idesc), "r"(acc)
                        : "memory");
                else
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                        "l"(a2), "l"(b2), "r"(idesc), "r"(acc)
                        : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&bar))
                         : "memory");
            // wait for this batch (bounded: about two seconds)
            const long long t0 = clock64();
            for (;;) {
                unsigned ok;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}"
                    : "=r"(ok)
                    : "r"(smem_addr(&bar)), "r"(phase)
                    : "memory");
                if (ok) break;
                if (clock64() - t0 > 4000000000LL) {
                    atomicExch(status, DEV_TC_WAIT);
                    break;
                }
            }
            phase ^= 1u;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem) : "memory");
    }
}

float time_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace
}  // namespace qsk

using namespace qsk;

extern "C" int qsk_measure_peaks(int device, double *out) {
    if (!out) return set_error(QSK_ERR_ARG, "null output");
    DeviceGuard dg(device);
    int sms = 0;
    QSK_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    DBuf<float> fo;
    DBuf<unsigned> uo;
    DBuf<int> st;
    QSK_CK(fo.alloc(PK_THREADS));
    QSK_CK(uo.alloc(PK_THREADS));
    QSK_CK(st.alloc(1));
    QSK_CK(cudaMemset(st.p, 0, sizeof(int)));
    cudaEvent_t e0, e1;
    QSK_CK(cudaEventCreate(&e0));
    QSK_CK(cudaEventCreate(&e1));
    const int blocks = sms * 8, iters = 256;
    const double ops = double(blocks) * PK_THREADS * iters * 16 * PK_CHAINS;
    // FP32 FMA (2 flops each)
    k_peak_ffma<<<blocks, PK_THREADS>>>(fo.p, 64, 0.999f, 1e-3f);
    QSK_CK(cudaEventRecord(e0));
    k_peak_ffma<<<blocks, PK_THREADS>>>(fo.p, iters, 0.999f, 1e-3f);
    QSK_CK(cudaEventRecord(e1));
    QSK_CK(cudaEventSynchronize(e1));
    out[0] = 2.0 * ops / (time_ms(e0, e1) * 1e-3) / 1e12;
    // LOP3 (one 32-bit logic op each)
    k_peak_lop3<<<blocks, PK_THREADS>>>(uo.p, 64, 0x5A5A5A5Au, 0x3C3C3C3Cu);
    QSK_CK(cudaEventRecord(e0));
    k_peak_lop3<<<blocks, PK_THREADS>>>(uo.p, iters, 0x5A5A5A5Au, 0x3C3C3C3Cu);
    QSK_CK(cudaEventRecord(e1));
    QSK_CK(cudaEventSynchronize(e1));
    out[1] = ops / (time_ms(e0, e1) * 1e-3) / 1e12;
    // tcgen05 dense MMA: BF16 (K = 16 per MMA) and FP8 E4M3 (K = 32); the
    // shared-memory request (more than half an SM's) keeps one CTA per SM
    const int smem = 120 * 1024;
    QSK_CK(cudaFuncSetAttribute(k_peak_mma<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    QSK_CK(cudaFuncSetAttribute(k_peak_mma<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const int miters = 100;
    for (int kind = 0; kind < 2; ++kind) {
        auto kern = kind == 0 ? k_peak_mma<0> : k_peak_mma<1>;
        kern<<<sms, 128, smem>>>(8, st.p);
        QSK_CK(cudaEventRecord(e0));
        kern<<<sms, 128, smem>>>(miters, st.p);
        QSK_CK(cudaEventRecord(e1));
        QSK_CK(cudaEventSynchronize(e1));
        const double kmma = kind == 0 ? 16.0 : 32.0;
        const double flops = double(sms) * miters * 64 * 2.0 * 128 * 256 * kmma;
        out[2 + kind] = flops / (time_ms(e0, e1) * 1e-3) / 1e12;
    }
    QSK_CK(cudaGetLastError());
    int status = 0;
    QSK_CK(cudaMemcpy(&status, st.p, sizeof(int), cudaMemcpyDeviceToHost));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status != DEV_OK) return set_error(QSK_ERR_DEVICE, "peak benchmark: device status %d", status);
    return QSK_OK;
}

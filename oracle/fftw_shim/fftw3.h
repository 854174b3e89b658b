/*
 * Test infrastructure only: a project-written stand-in for the single-precision
 * FFTW3 API subset that the G2S reference CPU path calls.  FFTW itself is not
 * installed in this image, so the reference sources under the G2S tree are
 * compiled against this header and linked with fftw_shim.c to build the CPU
 * oracle / CPU baseline (never the GPU product).
 *
 * Call sites served (G2S paths):
 *   src/CPUThreadDevice.cpp:99-141  (plan_dft_c2r, plan_dft_r2c, plan_many_dft,
 *                                     plan_with_nthreads)
 *   src/CPUThreadDevice.cpp:204-207 (plan_dft_r2c, execute, destroy_plan)
 *   src/CPUThreadDevice.cpp:417-422,451 (execute, execute_dft_c2r)
 *   src/qs.cpp:967,2295             (init_threads, cleanup_threads)
 *
 * Semantics follow the published FFTW3 interface: unnormalised transforms,
 * row-major multi-dimensional arrays with the last dimension halved
 * (n/2+1 complex) for r2c/c2r, forward sign -1.
 */
#ifndef G2S_B200_FFTW_SHIM_H
#define G2S_B200_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float fftwf_complex[2];
typedef struct g2s_shim_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PATIENT (1U << 5)
#define FFTW_ESTIMATE (1U << 6)

fftwf_plan fftwf_plan_dft_r2c(int rank, const int *n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r(int rank, const int *n, fftwf_complex *in, float *out, unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany,
                               fftwf_complex *in, const int *inembed, int istride, int idist,
                               fftwf_complex *out, const int *onembed, int ostride, int odist,
                               int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex *in, float *out);
void fftwf_execute_dft_r2c(const fftwf_plan p, float *in, fftwf_complex *out);
void fftwf_destroy_plan(fftwf_plan p);
void fftwf_plan_with_nthreads(int nthreads);
int fftwf_init_threads(void);
void fftwf_cleanup_threads(void);

#ifdef __cplusplus
}
#endif

#endif

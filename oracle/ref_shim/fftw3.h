/*
 * fftw3.h stand-in used ONLY to compile the reference's own sources for
 * parity checks (FFTW3f is not installed on these machines).  Declares the
 * single-precision FFTW entry points the reference calls
 * (dedispersion/msosm/msosm_prepare.cpp:65-81,
 * simulated_pulsar/simulated_complex_signal.cpp:253-273) and implements them
 * in fftw3_shim.c on top of the oracle's FP64 FFT (results rounded to float).
 */
#ifndef MSOSM_REF_SHIM_FFTW3_H
#define MSOSM_REF_SHIM_FFTW3_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
#ifdef __cplusplus
}
#endif
#endif

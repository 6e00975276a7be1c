/*
 * fft_cpu.h -- FP64 complex DFT used by the oracle (test infrastructure only).
 *
 * This is the CPU transform behind the oracle restatement (atus_oracle.c) and
 * behind the FFTW-API shim (shim/fftw_shim.c) that lets the reference's own
 * programs build without FFTW.  It computes the same unnormalised transform
 * FFTW 3.3.8 computes for fftw_plan_dft_{1,2,3}d (reference call sites:
 * source/libs/lib_myutils/cft_1d.cpp:44-45, cft_2d.cpp:41-42, cft_3d.cpp:41-42):
 *
 *     out[k] = sum_j in[j] * exp(sign * 2*pi*i * j.k / n),  sign = -1 forward, +1 backward
 *
 * over a row-major array whose last index is contiguous.  Nothing on the
 * product path links this file.
 */
#ifndef ORACLE_FFT_CPU_H
#define ORACLE_FFT_CPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_fft_plan orc_fft_plan;

/* rank 1..3, n[0] slowest axis.  sign -1 forward, +1 backward. */
orc_fft_plan *orc_fft_plan_create(int rank, const int *n, int sign);
void orc_fft_plan_destroy(orc_fft_plan *p);
/* In-place transform of interleaved (re,im) doubles. */
void orc_fft_execute(const orc_fft_plan *p, double *data);
/* Number of OpenMP threads the transform uses (<=0: OpenMP default). */
void orc_fft_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif

/*
 * fftw3.h -- FFTW 3.3.8 API subset for building the reference programs in the
 * oracle (test infrastructure only; FFTW itself is not installed here).
 *
 * Declares exactly the FFTW entry points the reference's solver path uses
 * (source/libs/lib_myutils/cft_base.h:62-95, cft_{1,2,3}d.cpp constructors,
 * include/CSOB_Base.h:215-221, the programs' main()).  They are implemented in
 * fftw_shim.c on top of oracle/fft_cpu.c, which computes FFTW's unnormalised
 * c2c transform.  Only FFTW_ESTIMATE-style planning is offered: planning never
 * touches the arrays.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_1d(int n0, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);
double *fftw_alloc_real(size_t n);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif
#endif

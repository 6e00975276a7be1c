/*
 * fftw_shim.c -- FFTW API subset (see fftw3.h) on top of the oracle FFT.
 * Test infrastructure only.
 */
#include "fftw3.h"

#include <stdlib.h>
#include <string.h>

#include "../fft_cpu.h"

struct fftw_plan_s {
  orc_fft_plan *p;
  fftw_complex *in, *out;
  size_t n;
};

static fftw_plan make(int rank, const int *n, fftw_complex *in, fftw_complex *out, int sign) {
  struct fftw_plan_s *pl = (struct fftw_plan_s *)calloc(1, sizeof(*pl));
  pl->p = orc_fft_plan_create(rank, n, sign);
  pl->in = in;
  pl->out = out;
  pl->n = 1;
  for (int a = 0; a < rank; a++) pl->n *= (size_t)n[a];
  return pl;
}

fftw_plan fftw_plan_dft_1d(int n0, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  int n[1] = {n0};
  return make(1, n, in, out, sign);
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
  (void)flags;
  int n[2] = {n0, n1};
  return make(2, n, in, out, sign);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags) {
  (void)flags;
  int n[3] = {n0, n1, n2};
  return make(3, n, in, out, sign);
}
void fftw_execute(const fftw_plan pl) {
  if (pl->in != pl->out) memcpy(pl->out, pl->in, sizeof(fftw_complex) * pl->n);
  orc_fft_execute(pl->p, (double *)pl->out);
}
void fftw_destroy_plan(fftw_plan pl) {
  if (!pl) return;
  orc_fft_plan_destroy(pl->p);
  free(pl);
}
void *fftw_malloc(size_t n) {
  void *p = NULL;
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
  return p;
}
void fftw_free(void *p) { free(p); }
fftw_complex *fftw_alloc_complex(size_t n) { return (fftw_complex *)fftw_malloc(sizeof(fftw_complex) * n); }
double *fftw_alloc_real(size_t n) { return (double *)fftw_malloc(sizeof(double) * n); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { orc_fft_set_threads(nthreads); }
void fftw_cleanup_threads(void) {}
void fftw_cleanup(void) {}

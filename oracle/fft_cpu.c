/*
 * fft_cpu.c -- FP64 complex DFT for the oracle (test infrastructure only).
 *
 * Power-of-two lengths use an out-of-place Stockham radix-4 transform (with
 * one radix-2 pass when log2(n) is odd); other lengths fall back to a direct
 * O(n^2) sum, which the tests only use on small grids.  Twiddles
 * exp(sign*2*pi*i*k/n) are evaluated in long double and rounded once, with the
 * quarter-turn points set exactly.  Multi-dimensional transforms run axis by
 * axis over pencils, OpenMP-parallel over pencil groups; strided axes gather
 * PB pencils that are adjacent in memory so each gathered cache line is used
 * completely.
 *
 * Transform definition: FFTW 3.3.8 fftw_plan_dft_{1,2,3}d as called from
 * source/libs/lib_myutils/cft_{1,2,3}d.cpp (unnormalised, row-major).
 */
#include "fft_cpu.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#else
static int omp_get_max_threads(void) { return 1; }
#endif

#define PB 8 /* pencils gathered together on a strided axis */

struct orc_fft_plan {
  int rank;
  int n[3];
  int sign;
  double *tw[3]; /* per axis: 2*n doubles, exp(sign*2*pi*i*k/n) */
};

static int g_threads = 0;

void orc_fft_set_threads(int nthreads) { g_threads = nthreads; }

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void make_twiddles(double *tw, int n, int sign) {
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < n; k++) {
    double c, s;
    if (k == 0) {
      c = 1.0; s = 0.0;
    } else if (4L * k == n) {
      c = 0.0; s = 1.0;
    } else if (2L * k == n) {
      c = -1.0; s = 0.0;
    } else if (4L * k == 3L * n) {
      c = 0.0; s = -1.0;
    } else {
      long double th = two_pi * (long double)k / (long double)n;
      c = (double)cosl(th);
      s = (double)sinl(th);
    }
    tw[2 * k] = c;
    tw[2 * k + 1] = (double)sign * s;
  }
}

orc_fft_plan *orc_fft_plan_create(int rank, const int *n, int sign) {
  if (rank < 1 || rank > 3) return NULL;
  orc_fft_plan *p = (orc_fft_plan *)calloc(1, sizeof(orc_fft_plan));
  p->rank = rank;
  p->sign = sign < 0 ? -1 : 1;
  for (int a = 0; a < rank; a++) {
    p->n[a] = n[a];
    p->tw[a] = (double *)malloc(sizeof(double) * 2 * (size_t)n[a]);
    make_twiddles(p->tw[a], n[a], p->sign);
  }
  return p;
}

void orc_fft_plan_destroy(orc_fft_plan *p) {
  if (!p) return;
  for (int a = 0; a < p->rank; a++) free(p->tw[a]);
  free(p);
}

/* One pencil, power of two: Stockham radix-4 (+ one radix-2).  x holds the
 * input, y is scratch; the result is left in x. */
static void pencil_pow2(double *x, double *y, int n, const double *tw, int sign) {
  if (n == 1) return;
  double *src = x, *dst = y;
  int Ns = 1;
  const int n4 = n / 4;
  while (Ns * 4 <= n) {
    const int stride = n / (4 * Ns); /* twiddle index step */
    for (int j = 0; j < n4; j++) {
      const int k = j & (Ns - 1);
      double ar[4], ai[4];
      for (int r = 0; r < 4; r++) {
        const double vr = src[2 * (j + r * n4)], vi = src[2 * (j + r * n4) + 1];
        if (r == 0 || k == 0) {
          ar[r] = vr; ai[r] = vi;
        } else {
          const int m = r * k * stride;
          const double wr = tw[2 * m], wi = tw[2 * m + 1];
          ar[r] = vr * wr - vi * wi;
          ai[r] = vr * wi + vi * wr;
        }
      }
      const double t0r = ar[0] + ar[2], t0i = ai[0] + ai[2];
      const double t1r = ar[0] - ar[2], t1i = ai[0] - ai[2];
      const double t2r = ar[1] + ar[3], t2i = ai[1] + ai[3];
      /* (a1 - a3) * (sign * i) */
      const double dr = ar[1] - ar[3], di = ai[1] - ai[3];
      const double t3r = -(double)sign * di, t3i = (double)sign * dr;
      const int base = (j / Ns) * Ns * 4 + k;
      dst[2 * base] = t0r + t2r;               dst[2 * base + 1] = t0i + t2i;
      dst[2 * (base + Ns)] = t1r + t3r;        dst[2 * (base + Ns) + 1] = t1i + t3i;
      dst[2 * (base + 2 * Ns)] = t0r - t2r;    dst[2 * (base + 2 * Ns) + 1] = t0i - t2i;
      dst[2 * (base + 3 * Ns)] = t1r - t3r;    dst[2 * (base + 3 * Ns) + 1] = t1i - t3i;
    }
    double *t = src; src = dst; dst = t;
    Ns *= 4;
  }
  if (Ns < n) { /* one radix-2 pass, Ns == n/2 */
    const int n2 = n / 2;
    const int stride = n / (2 * Ns);
    for (int j = 0; j < n2; j++) {
      const int k = j & (Ns - 1);
      const double ar = src[2 * j], ai = src[2 * j + 1];
      double br = src[2 * (j + n2)], bi = src[2 * (j + n2) + 1];
      if (k != 0) {
        const int m = k * stride;
        const double wr = tw[2 * m], wi = tw[2 * m + 1];
        const double tr = br * wr - bi * wi;
        bi = br * wi + bi * wr;
        br = tr;
      }
      const int base = (j / Ns) * Ns * 2 + k;
      dst[2 * base] = ar + br;        dst[2 * base + 1] = ai + bi;
      dst[2 * (base + Ns)] = ar - br; dst[2 * (base + Ns) + 1] = ai - bi;
    }
    double *t = src; src = dst; dst = t;
  }
  if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

/* One pencil, any length: direct sum (small test grids only). */
static void pencil_direct(double *x, double *y, int n, const double *tw) {
  for (int k = 0; k < n; k++) {
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < n; j++) {
      const long m = ((long)j * (long)k) % n;
      const double wr = tw[2 * m], wi = tw[2 * m + 1];
      sr += x[2 * j] * wr - x[2 * j + 1] * wi;
      si += x[2 * j] * wi + x[2 * j + 1] * wr;
    }
    y[2 * k] = sr;
    y[2 * k + 1] = si;
  }
  memcpy(x, y, sizeof(double) * 2 * (size_t)n);
}

static void pencil(double *x, double *y, int n, const double *tw, int sign) {
  if (is_pow2(n)) pencil_pow2(x, y, n, tw, sign);
  else pencil_direct(x, y, n, tw);
}

/* Transform every pencil along one axis of a row-major [outer][n][inner] array. */
static void axis_pass(double *data, long outer, int n, long inner, const double *tw, int sign) {
  if (n == 1) return;
  if (inner == 1) {
    #pragma omp parallel num_threads(g_threads > 0 ? g_threads : omp_get_max_threads())
    {
      double *scratch = (double *)malloc(sizeof(double) * 2 * (size_t)n);
      #pragma omp for schedule(static)
      for (long o = 0; o < outer; o++)
        pencil(data + 2 * o * (long)n, scratch, n, tw, sign);
      free(scratch);
    }
    return;
  }
  const long groups_per_outer = (inner + PB - 1) / PB;
  const long ngroups = outer * groups_per_outer;
  #pragma omp parallel num_threads(g_threads > 0 ? g_threads : omp_get_max_threads())
  {
    double *buf = (double *)malloc(sizeof(double) * 2 * (size_t)n * PB);
    double *scratch = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    #pragma omp for schedule(static)
    for (long g = 0; g < ngroups; g++) {
      const long o = g / groups_per_outer;
      const long i0 = (g % groups_per_outer) * PB;
      const int nb = (int)((inner - i0) < PB ? (inner - i0) : PB);
      double *base = data + 2 * (o * (long)n * inner + i0);
      for (int j = 0; j < n; j++) {
        const double *row = base + 2 * (long)j * inner;
        for (int b = 0; b < nb; b++) {
          buf[2 * ((long)b * n + j)] = row[2 * b];
          buf[2 * ((long)b * n + j) + 1] = row[2 * b + 1];
        }
      }
      for (int b = 0; b < nb; b++) pencil(buf + 2 * (long)b * n, scratch, n, tw, sign);
      for (int j = 0; j < n; j++) {
        double *row = base + 2 * (long)j * inner;
        for (int b = 0; b < nb; b++) {
          row[2 * b] = buf[2 * ((long)b * n + j)];
          row[2 * b + 1] = buf[2 * ((long)b * n + j) + 1];
        }
      }
    }
    free(buf);
    free(scratch);
  }
}

void orc_fft_execute(const orc_fft_plan *p, double *data) {
  long total = 1;
  for (int a = 0; a < p->rank; a++) total *= p->n[a];
  /* Innermost axis first; the order of separable 1D passes does not change
   * the exact result, only the rounding. */
  for (int a = p->rank - 1; a >= 0; a--) {
    long inner = 1;
    for (int b = a + 1; b < p->rank; b++) inner *= p->n[b];
    const long outer = total / (inner * p->n[a]);
    axis_pass(data, outer, p->n[a], inner, p->tw[a], p->sign);
  }
}

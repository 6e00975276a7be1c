/*
 * gsl_shim_types.h -- the GSL 2.5 types and routines that
 * CRT_Base_IF::Numerical_Bragg / Numerical_Raman use (include/CRT_Base_IF.h:
 * 426-632), for building the reference programs in the oracle (test
 * infrastructure only; GSL itself is not installed here).
 *
 * gsl_eigen_hermv is a cyclic complex Jacobi eigensolver (each (p,q) rotation
 * first rotates the phase of A_pq away, then applies the real symmetric Jacobi
 * rotation); it returns eigenvalues unordered and orthonormal eigenvectors in
 * the columns of evec, as GSL documents.  zgemm/zgemv are the textbook loops.
 */
#ifndef ORACLE_SHIM_GSL_TYPES_H
#define ORACLE_SHIM_GSL_TYPES_H
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double dat[2]; } gsl_complex;
typedef struct { size_t size1, size2; gsl_complex *data; } gsl_matrix_complex;
typedef struct { size_t size; double *data; } gsl_vector;
typedef struct { size_t size; gsl_complex *data; } gsl_vector_complex;
typedef struct { size_t n; } gsl_eigen_hermv_workspace;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE_t;

static inline gsl_complex gsl_complex_rect(double x, double y) { gsl_complex z; z.dat[0] = x; z.dat[1] = y; return z; }
#define GSL_COMPLEX_ONE (gsl_complex_rect(1.0, 0.0))
#define GSL_COMPLEX_ZERO (gsl_complex_rect(0.0, 0.0))

static inline void gsl_shim_range(size_t i, size_t n) {
  if (i >= n) { fprintf(stderr, "gsl shim: index out of range\n"); abort(); }
}
static inline gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2) {
  gsl_matrix_complex *m = (gsl_matrix_complex *)malloc(sizeof(*m));
  m->size1 = n1; m->size2 = n2;
  m->data = (gsl_complex *)malloc(sizeof(gsl_complex) * n1 * n2);
  return m;
}
static inline gsl_matrix_complex *gsl_matrix_complex_calloc(size_t n1, size_t n2) {
  gsl_matrix_complex *m = gsl_matrix_complex_alloc(n1, n2);
  memset(m->data, 0, sizeof(gsl_complex) * n1 * n2);
  return m;
}
static inline void gsl_matrix_complex_free(gsl_matrix_complex *m) { if (m) { free(m->data); free(m); } }
static inline void gsl_matrix_complex_set_zero(gsl_matrix_complex *m) {
  memset(m->data, 0, sizeof(gsl_complex) * m->size1 * m->size2);
}
static inline void gsl_matrix_complex_set(gsl_matrix_complex *m, size_t i, size_t j, gsl_complex z) {
  gsl_shim_range(i, m->size1); gsl_shim_range(j, m->size2);
  m->data[i * m->size2 + j] = z;
}
static inline gsl_complex gsl_matrix_complex_get(const gsl_matrix_complex *m, size_t i, size_t j) {
  gsl_shim_range(i, m->size1); gsl_shim_range(j, m->size2);
  return m->data[i * m->size2 + j];
}
static inline gsl_vector *gsl_vector_alloc(size_t n) {
  gsl_vector *v = (gsl_vector *)malloc(sizeof(*v));
  v->size = n; v->data = (double *)calloc(n, sizeof(double));
  return v;
}
static inline void gsl_vector_free(gsl_vector *v) { if (v) { free(v->data); free(v); } }
static inline double gsl_vector_get(const gsl_vector *v, size_t i) { gsl_shim_range(i, v->size); return v->data[i]; }
static inline gsl_vector_complex *gsl_vector_complex_alloc(size_t n) {
  gsl_vector_complex *v = (gsl_vector_complex *)malloc(sizeof(*v));
  v->size = n; v->data = (gsl_complex *)calloc(n, sizeof(gsl_complex));
  return v;
}
static inline void gsl_vector_complex_free(gsl_vector_complex *v) { if (v) { free(v->data); free(v); } }
static inline void gsl_vector_complex_set(gsl_vector_complex *v, size_t i, gsl_complex z) {
  gsl_shim_range(i, v->size); v->data[i] = z;
}
static inline gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i) {
  gsl_shim_range(i, v->size); return v->data[i];
}
static inline gsl_eigen_hermv_workspace *gsl_eigen_hermv_alloc(size_t n) {
  gsl_eigen_hermv_workspace *w = (gsl_eigen_hermv_workspace *)malloc(sizeof(*w));
  w->n = n;
  return w;
}
static inline void gsl_eigen_hermv_free(gsl_eigen_hermv_workspace *w) { free(w); }

/* A is destroyed (GSL also destroys it). */
static inline int gsl_eigen_hermv(gsl_matrix_complex *Am, gsl_vector *eval, gsl_matrix_complex *evec,
                                  gsl_eigen_hermv_workspace *w) {
  const size_t n = w->n;
  gsl_complex *A = Am->data, *V = evec->data;
#define AR(i, j) A[(i) * n + (j)].dat[0]
#define AI(i, j) A[(i) * n + (j)].dat[1]
#define VR(i, j) V[(i) * n + (j)].dat[0]
#define VI(i, j) V[(i) * n + (j)].dat[1]
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j < n; j++) { VR(i, j) = (i == j) ? 1.0 : 0.0; VI(i, j) = 0.0; }
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0;
    for (size_t p = 0; p < n; p++)
      for (size_t q = p + 1; q < n; q++) off += AR(p, q) * AR(p, q) + AI(p, q) * AI(p, q);
    if (off == 0.0) break;
    for (size_t p = 0; p < n; p++) {
      for (size_t q = p + 1; q < n; q++) {
        const double mag = hypot(AR(p, q), AI(p, q));
        if (mag == 0.0) continue;
        /* phase: column q *= e^{-i phi}, row q *= e^{+i phi} -> A_pq real */
        const double er = AR(p, q) / mag, ei = AI(p, q) / mag; /* e^{i phi} */
        for (size_t k = 0; k < n; k++) {
          double r = AR(k, q), im = AI(k, q);
          AR(k, q) = r * er + im * ei; AI(k, q) = im * er - r * ei;
          r = VR(k, q); im = VI(k, q);
          VR(k, q) = r * er + im * ei; VI(k, q) = im * er - r * ei;
        }
        for (size_t k = 0; k < n; k++) {
          const double r = AR(q, k), im = AI(q, k);
          AR(q, k) = r * er - im * ei; AI(q, k) = im * er + r * ei;
        }
        const double app = AR(p, p), aqq = AR(q, q), apq = AR(p, q);
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (size_t k = 0; k < n; k++) { /* columns p, q */
          const double pr = AR(k, p), pi = AI(k, p), qr = AR(k, q), qi = AI(k, q);
          AR(k, p) = c * pr - s * qr; AI(k, p) = c * pi - s * qi;
          AR(k, q) = s * pr + c * qr; AI(k, q) = s * pi + c * qi;
          const double vpr = VR(k, p), vpi = VI(k, p), vqr = VR(k, q), vqi = VI(k, q);
          VR(k, p) = c * vpr - s * vqr; VI(k, p) = c * vpi - s * vqi;
          VR(k, q) = s * vpr + c * vqr; VI(k, q) = s * vpi + c * vqi;
        }
        for (size_t k = 0; k < n; k++) { /* rows p, q */
          const double pr = AR(p, k), pi = AI(p, k), qr = AR(q, k), qi = AI(q, k);
          AR(p, k) = c * pr - s * qr; AI(p, k) = c * pi - s * qi;
          AR(q, k) = s * pr + c * qr; AI(q, k) = s * pi + c * qi;
        }
        AR(p, q) = AI(p, q) = AR(q, p) = AI(q, p) = 0.0;
      }
    }
  }
  for (size_t i = 0; i < n; i++) eval->data[i] = AR(i, i);
#undef AR
#undef AI
#undef VR
#undef VI
  return 0;
}

static inline gsl_complex gsl_shim_op(const gsl_matrix_complex *M, CBLAS_TRANSPOSE_t t, size_t i, size_t j) {
  if (t == CblasNoTrans) return M->data[i * M->size2 + j];
  gsl_complex z = M->data[j * M->size2 + i];
  if (t == CblasConjTrans) z.dat[1] = -z.dat[1];
  return z;
}
static inline int gsl_blas_zgemm(CBLAS_TRANSPOSE_t ta, CBLAS_TRANSPOSE_t tb, const gsl_complex alpha,
                                 const gsl_matrix_complex *A, const gsl_matrix_complex *B,
                                 const gsl_complex beta, gsl_matrix_complex *C) {
  const size_t M = C->size1, N = C->size2, K = (ta == CblasNoTrans) ? A->size2 : A->size1;
  for (size_t i = 0; i < M; i++)
    for (size_t j = 0; j < N; j++) {
      double sr = 0, si = 0;
      for (size_t k = 0; k < K; k++) {
        const gsl_complex a = gsl_shim_op(A, ta, i, k), b = gsl_shim_op(B, tb, k, j);
        sr += a.dat[0] * b.dat[0] - a.dat[1] * b.dat[1];
        si += a.dat[0] * b.dat[1] + a.dat[1] * b.dat[0];
      }
      gsl_complex *c = &C->data[i * N + j];
      const double cr = c->dat[0], ci = c->dat[1];
      c->dat[0] = alpha.dat[0] * sr - alpha.dat[1] * si + beta.dat[0] * cr - beta.dat[1] * ci;
      c->dat[1] = alpha.dat[0] * si + alpha.dat[1] * sr + beta.dat[0] * ci + beta.dat[1] * cr;
    }
  return 0;
}
static inline int gsl_blas_zgemv(CBLAS_TRANSPOSE_t ta, const gsl_complex alpha, const gsl_matrix_complex *A,
                                 const gsl_vector_complex *x, const gsl_complex beta, gsl_vector_complex *y) {
  const size_t M = y->size, K = x->size;
  for (size_t i = 0; i < M; i++) {
    double sr = 0, si = 0;
    for (size_t k = 0; k < K; k++) {
      const gsl_complex a = gsl_shim_op(A, ta, i, k), b = x->data[k];
      sr += a.dat[0] * b.dat[0] - a.dat[1] * b.dat[1];
      si += a.dat[0] * b.dat[1] + a.dat[1] * b.dat[0];
    }
    const double yr = y->data[i].dat[0], yi = y->data[i].dat[1];
    y->data[i].dat[0] = alpha.dat[0] * sr - alpha.dat[1] * si + beta.dat[0] * yr - beta.dat[1] * yi;
    y->data[i].dat[1] = alpha.dat[0] * si + alpha.dat[1] * sr + beta.dat[0] * yi + beta.dat[1] * yr;
  }
  return 0;
}
#endif

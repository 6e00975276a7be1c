/*
 * atus_oracle.c -- CPU restatement of ATUS-2's split-step / Sobolev hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is compared
 * against; nothing shipped links or calls it.  Only tests/, the smoke check and
 * bench.py's CPU-baseline leg load it (through oracle/oracle.py).
 *
 * Every routine restates one reference routine (paths relative to the ATUS-2
 * tree) with the same floating-point operation order, so that, single-threaded
 * and built with -ffp-contract=off, it reproduces the reference program
 * compiled from its own sources (oracle/_ref) bit for bit:
 *
 *   orc_get_x / orc_get_k     cft_1d.cpp:85-108, cft_2d.cpp:81-113, cft_3d.cpp:128-166
 *                             (wrapped k, because CRT_Base::Allocate calls SetFix(false),
 *                             include/CRT_Base.h:195)
 *   ft()                      cft_1d.cpp:61-77 + scale :191-201; cft_2d.cpp:58-74 +
 *                             scale :449-459; cft_3d.cpp:58-74 + scale :627-637
 *   orc_set_dt (tables)       include/CRT_Base.h:252-274 (Init); CRT_Base_2.h:194-221
 *   orc_ft_step               include/CRT_Base.h:336-392 (Do_FT_Step_full/half)
 *   orc_nl_step               include/CRT_Base.h:396-441 (Do_NL_Step)
 *   orc_nl_if_step            include/CRT_Base_IF.h:380-419 (freeprop of the IF programs)
 *   orc_bragg_ad              source/interferometry/src/bragg.cpp:185-304 (Do_Bragg_ad)
 *   orc_double_bragg_ad       source/interferometry/src/double_bragg.cpp:100-258
 *                             (Bragg_double::Do_Double_Bragg_ad)
 *   orc_nl_if2_step           include/CRT_Base_IF_2.h:378-416 (freeprop of the
 *                             two-species programs)
 *   orc_bragg_ds_ad           source/interferometry/src/bragg_ds.cpp:111-322
 *                             (Bragg_single::Do_Bragg_ad of bragg_ds)
 *   orc_rabi_integrals_comp   include/CRT_Base_IF_2.h:115-210 (species 2 on
 *                             component no_int_states/2)
 *   orc_numerical_bragg       include/CRT_Base_IF.h:426-526 (Numerical_Bragg)
 *   orc_numerical_raman       include/CRT_Base_IF.h:533-632 (Numerical_Raman)
 *                             Both call the GSL routines the reference calls;
 *                             GSL is not installed here, so they come from the
 *                             same shim the reference programs in oracle/_ref
 *                             are built against (shim/gsl/gsl_shim_types.h).
 *   orc_block                 include/CRT_Base.h:776-786 / CRT_Base_IF.h:779-789
 *   orc_particle_number       include/CRT_Base.h:586-599
 *   orc_expval_position/momentum include/CRT_Base.h:480-580
 *   orc_setup_momentum        include/CRT_Base.h:448-473
 *   orc_rabi_integrals        include/CRT_Base_IF.h:207-281
 *   orc_sob_*                 include/CSOB_Base.h:228-543 (Init, Compute_*, Project,
 *                             Compute_res, run, Renormalize_All_Psi); orc_sob_mu follows
 *                             the formula of Compute_mu (:399-424) with m_ar as the
 *                             volume element.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fft_cpu.h"
#include "shim/gsl/gsl_shim_types.h"
#include <omp.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ORC_MAXC 4

typedef struct {
  double beta[3];
  double DeltaL[ORC_MAXC];
  double Amp[2];
  double laser_k[2];
  double laser_dk[2];
  double laser_domh[2];
  double phase[2];
  double chirp_rate[2];
  double chirp;
} orc_laser;

typedef struct {
  int dim;
  int ncomp;
  long n[3];      /* nDimX, nDimY, nDimZ (1 for unused axes) */
  double d[3];    /* dx, dy, dz */
  double dk[3];   /* dkx, dky, dkz */
  long npts;
  int shift[3];
  double ar, ar_k;
  double t, dt;
  double alpha[ORC_MAXC][3];
  double gs[ORC_MAXC * ORC_MAXC];
  double *psi[ORC_MAXC];
  double *V[ORC_MAXC];  /* NULL: no potential (m_potenial_initialized == false) */
  double *half[ORC_MAXC], *full[ORC_MAXC]; /* kinetic tables, shared between equal alphas */
  orc_fft_plan *fwd, *bwd;
  /* Sobolev state */
  double *lap[ORC_MAXC], *sob[ORC_MAXC], *grad[ORC_MAXC];
  double *op[ORC_MAXC], *op2[ORC_MAXC];
  double stepsize;
  /* second species of the two-species programs and the pulse windows of
   * their bragg_ad (seq.time, seq.duration[0..1]) */
  orc_laser L2;
  double win_t0, win_dur[2];
} orc_ctx;

/* ------------------------------------------------------------------ grid */

static void get_idx(const orc_ctx *c, long l, long *i, long *j, long *k) {
  if (c->dim == 1) { *i = l; *j = 0; *k = 0; }
  else if (c->dim == 2) { *i = l / c->n[1]; *j = l - *i * c->n[1]; *k = 0; }
  else {
    *i = l / c->n[1] / c->n[2];
    *j = (l - *i * c->n[1] * c->n[2]) / c->n[2];
    *k = l - *i * c->n[1] * c->n[2] - *j * c->n[2];
  }
}

void orc_get_x(const orc_ctx *c, long l, double *x) {
  long ijk[3];
  get_idx(c, l, &ijk[0], &ijk[1], &ijk[2]);
  for (int a = 0; a < c->dim; a++) x[a] = (double)(ijk[a] - c->shift[a]) * c->d[a];
}

void orc_get_k(const orc_ctx *c, long l, double *k) {
  long ijk[3];
  get_idx(c, l, &ijk[0], &ijk[1], &ijk[2]);
  for (int a = 0; a < c->dim; a++) {
    const long t = (ijk[a] + c->shift[a]) % c->n[a];
    k[a] = c->dk[a] * (double)(t - c->shift[a]);
  }
}

static void scale(const orc_ctx *c, double *data, const double *s) {
  double fak;
  if (c->dim == 1) fak = s[0] / sqrt(2.0 * M_PI);
  else if (c->dim == 2) fak = 0.5 * s[0] * s[1] / M_PI;
  else fak = s[0] * s[1] * s[2] / pow(2 * M_PI, 1.5);
  #pragma omp parallel for schedule(static)
  for (long i = 0; i < c->npts; i++) {
    data[2 * i] *= fak;
    data[2 * i + 1] *= fak;
  }
}

/* cft_Nd::ft with m_bfix == false: transform then scale. */
void orc_ft(orc_ctx *c, double *data, int isign) {
  if (isign == -1) {
    orc_fft_execute(c->fwd, data);
    scale(c, data, c->d);
  } else {
    orc_fft_execute(c->bwd, data);
    scale(c, data, c->dk);
  }
}

orc_ctx *orc_create(int dim, int ncomp, const long long *n, const double *d, const double *dk) {
  if (dim < 1 || dim > 3 || ncomp < 1 || ncomp > ORC_MAXC) return NULL;
  orc_ctx *c = (orc_ctx *)calloc(1, sizeof(orc_ctx));
  c->dim = dim;
  c->ncomp = ncomp;
  c->npts = 1;
  int nn[3];
  for (int a = 0; a < 3; a++) {
    c->n[a] = (a < dim) ? (long)n[a] : 1;
    c->d[a] = (a < dim) ? d[a] : 0.0;
    c->dk[a] = (a < dim) ? dk[a] : 0.0;
    c->shift[a] = (int)(c->n[a] / 2);
    nn[a] = (int)c->n[a];
    c->npts *= c->n[a];
  }
  /* m_ar and m_ar_k as CRT_shared::Read_header, include/CRT_shared.h:131-172 */
  if (dim == 1) { c->ar = c->d[0]; c->ar_k = c->dk[0]; }
  else if (dim == 2) { c->ar = c->d[0] * c->d[1]; c->ar_k = c->dk[0] * c->dk[1]; }
  else { c->ar = c->d[0] * c->d[1] * c->d[2]; c->ar_k = c->dk[0] * c->dk[1] * c->dk[2]; }
  c->fwd = orc_fft_plan_create(dim, nn, -1);
  c->bwd = orc_fft_plan_create(dim, nn, +1);
  for (int i = 0; i < ncomp; i++) c->psi[i] = (double *)calloc((size_t)c->npts * 2, sizeof(double));
  c->dt = 0.001;
  c->win_dur[0] = c->win_dur[1] = HUGE_VAL;
  return c;
}

static void free_tables(orc_ctx *c) {
  for (int i = 0; i < c->ncomp; i++) {
    int shared = 0;
    for (int j = 0; j < i; j++) if (c->half[j] == c->half[i]) shared = 1;
    if (!shared) { free(c->half[i]); free(c->full[i]); }
  }
  for (int i = 0; i < c->ncomp; i++) c->half[i] = c->full[i] = NULL;
}

void orc_destroy(orc_ctx *c) {
  if (!c) return;
  free_tables(c);
  for (int i = 0; i < c->ncomp; i++) {
    free(c->psi[i]); free(c->V[i]);
    free(c->lap[i]); free(c->sob[i]); free(c->grad[i]);
    free(c->op[i]); free(c->op2[i]);
  }
  orc_fft_plan_destroy(c->fwd);
  orc_fft_plan_destroy(c->bwd);
  free(c);
}

double *orc_psi(orc_ctx *c, int comp) { return c->psi[comp]; }
long orc_npts(const orc_ctx *c) { return c->npts; }
double orc_get_t(const orc_ctx *c) { return c->t; }
void orc_set_t(orc_ctx *c, double t) { c->t = t; }
void orc_set_gs(orc_ctx *c, const double *gs) {
  memcpy(c->gs, gs, sizeof(double) * c->ncomp * c->ncomp);
}
void orc_set_alpha(orc_ctx *c, int comp, const double *alpha) {
  for (int a = 0; a < 3; a++) c->alpha[comp][a] = (a < c->dim) ? alpha[a] : 0.0;
}
/* V == NULL clears the potential for that component. */
void orc_set_potential(orc_ctx *c, int comp, const double *V) {
  if (!V) { free(c->V[comp]); c->V[comp] = NULL; return; }
  if (!c->V[comp]) c->V[comp] = (double *)malloc(sizeof(double) * c->npts);
  memcpy(c->V[comp], V, sizeof(double) * c->npts);
}

/* Kinetic tables, CRT_Base::Init (include/CRT_Base.h:252-274):
 * phi = (-dt) * (k.scale(alpha) * k);  half = e^{i phi/2}, full = e^{i phi}. */
void orc_set_dt(orc_ctx *c, double dt) {
  c->dt = dt;
  free_tables(c);
  for (int i = 0; i < c->ncomp; i++) {
    int src = -1;
    for (int j = 0; j < i; j++)
      if (memcmp(c->alpha[j], c->alpha[i], sizeof(c->alpha[i])) == 0) { src = j; break; }
    if (src >= 0) { c->half[i] = c->half[src]; c->full[i] = c->full[src]; continue; }
    double *h = (double *)malloc(sizeof(double) * 2 * c->npts);
    double *f = (double *)malloc(sizeof(double) * 2 * c->npts);
    const double mdt = -dt;
    #pragma omp parallel for schedule(static)
    for (long l = 0; l < c->npts; l++) {
      double k[3];
      orc_get_k(c, l, k);
      double dot = 0;
      for (int a = 0; a < c->dim; a++) dot += (k[a] * c->alpha[i][a]) * k[a];
      const double phi = mdt * dot;
      h[2 * l] = cos(0.5 * phi);
      h[2 * l + 1] = sin(0.5 * phi);
      f[2 * l] = cos(phi);
      f[2 * l + 1] = sin(phi);
    }
    c->half[i] = h;
    c->full[i] = f;
  }
}

/* --------------------------------------------------------- split steps */

void orc_ft_step(orc_ctx *c, int half) {
  for (int i = 0; i < c->ncomp; i++) orc_ft(c, c->psi[i], -1);
  for (int i = 0; i < c->ncomp; i++) {
    double *P = c->psi[i];
    const double *T = half ? c->half[i] : c->full[i];
    #pragma omp parallel for schedule(static)
    for (long l = 0; l < c->npts; l++) {
      const double tmp1 = P[2 * l];
      P[2 * l] = P[2 * l] * T[2 * l] - P[2 * l + 1] * T[2 * l + 1];
      P[2 * l + 1] = P[2 * l + 1] * T[2 * l] + tmp1 * T[2 * l + 1];
    }
  }
  for (int i = 0; i < c->ncomp; i++) orc_ft(c, c->psi[i], +1);
  if (half) c->t += 0.5 * c->dt;
  else c->t += c->dt;
}

static void apply_phases(orc_ctx *c, long l, const double *phi) {
  for (int i = 0; i < c->ncomp; i++) {
    double im1, re1;
    sincos(phi[i], &im1, &re1);
    double *P = c->psi[i];
    const double tmp1 = P[2 * l];
    P[2 * l] = P[2 * l] * re1 - P[2 * l + 1] * im1;
    P[2 * l + 1] = P[2 * l + 1] * re1 + tmp1 * im1;
  }
}

void orc_nl_step(orc_ctx *c) {
  const double dt = -c->dt;
  const int n = c->ncomp;
  #pragma omp parallel for schedule(static)
  for (long l = 0; l < c->npts; l++) {
    double phi[ORC_MAXC];
    for (int i = 0; i < n; i++) {
      phi[i] = c->V[i] ? c->V[i][l] : 0.0;
      for (int j = 0; j < n; j++) {
        const double *P = c->psi[j];
        phi[i] += c->gs[j + n * i] * (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
      }
      phi[i] *= dt;
    }
    apply_phases(c, l, phi);
  }
}

void orc_nl_if_step(orc_ctx *c, const orc_laser *L) {
  const double dt = -c->dt;
  const int n = c->ncomp;
  #pragma omp parallel for schedule(static)
  for (long l = 0; l < c->npts; l++) {
    double phi[ORC_MAXC];
    for (int i = 0; i < n; i++) {
      phi[i] = 0;
      for (int j = 0; j < n; j++) {
        const double *P = c->psi[j];
        phi[i] += c->gs[j + n * i] * (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
      }
      double x[3];
      orc_get_x(c, l, x);
      phi[i] += L->beta[0] * x[0] - L->DeltaL[i];
      phi[i] *= dt;
    }
    apply_phases(c, l, phi);
  }
}

void orc_bragg_ad(orc_ctx *c, const orc_laser *L, double F) {
  const double dt = c->dt;
  const double t1 = c->t + 0.5 * dt;
  double *P1 = c->psi[0], *P2 = c->psi[1];
  const double *gs = c->gs;
  #pragma omp parallel for schedule(static)
  for (long l = 0; l < c->npts; l++) {
    double x[3];
    orc_get_x(c, l, x);
    double tmp1 = P1[2 * l] * P1[2 * l] + P1[2 * l + 1] * P1[2 * l + 1];
    double tmp2 = P2[2 * l] * P2[2 * l] + P2[2 * l + 1] * P2[2 * l + 1];
    const double V11 = gs[0] * tmp1 + gs[1] * tmp2 + L->beta[0] * x[0];
    const double V22 = gs[2] * tmp1 + gs[3] * tmp2 - L->DeltaL[1] + L->beta[0] * x[0];
    const double Omega = F * L->Amp[0] *
        cos(L->laser_k[0] * x[0] - (L->laser_domh[0] + L->chirp * t1 + L->chirp_rate[0] * t1) * t1 +
            L->phase[0] / 2);
    double re1, im1;
    if (Omega == 0.0) {
      sincos(-dt * V11, &im1, &re1);
      tmp1 = P1[2 * l];
      P1[2 * l] = tmp1 * re1 - P1[2 * l + 1] * im1;
      P1[2 * l + 1] = tmp1 * im1 + P1[2 * l + 1] * re1;
      sincos(-dt * V22, &im1, &re1);
      tmp1 = P2[2 * l];
      P2[2 * l] = tmp1 * re1 - P2[2 * l + 1] * im1;
      P2[2 * l + 1] = tmp1 * im1 + P2[2 * l + 1] * re1;
      continue;
    }
    double eta[2], gp[2], gm[2], O11[2], O12[2], O21[2], O22[2];
    sincos(-0.5 * (L->laser_dk[0] * x[0]), &im1, &re1);
    eta[0] = re1;
    eta[1] = im1;
    tmp1 = sqrt((V11 - V22) * (V11 - V22) + 4.0 * Omega * Omega);
    const double Ep = 0.5 * (V11 + V22 + tmp1);
    const double Em = 0.5 * (V11 + V22 - tmp1);
    sincos(-dt * Ep, &im1, &re1);
    tmp1 = 1.0 / fabs((V11 - Ep) * (V11 - Ep) + Omega * Omega);
    gp[0] = tmp1 * re1;
    gp[1] = tmp1 * im1;
    sincos(-dt * Em, &im1, &re1);
    tmp1 = 1.0 / fabs((V11 - Em) * (V11 - Em) + Omega * Omega);
    gm[0] = tmp1 * re1;
    gm[1] = tmp1 * im1;
    tmp1 = Omega * Omega;
    O11[0] = tmp1 * (gp[0] + gm[0]);
    O11[1] = tmp1 * (gp[1] + gm[1]);
    tmp1 = V11 - Ep;
    tmp2 = V11 - Em;
    O22[0] = tmp1 * tmp1 * gp[0] + tmp2 * tmp2 * gm[0];
    O22[1] = tmp1 * tmp1 * gp[1] + tmp2 * tmp2 * gm[1];
    O12[0] = -Omega * (tmp1 * gp[0] + tmp2 * gm[0]);
    O12[1] = -Omega * (tmp1 * gp[1] + tmp2 * gm[1]);
    O21[0] = O12[0];
    O21[1] = O12[1];
    tmp1 = O12[0];
    O12[0] = eta[0] * tmp1 - eta[1] * O12[1];
    O12[1] = eta[1] * tmp1 + eta[0] * O12[1];
    tmp1 = O21[0];
    O21[0] = eta[0] * tmp1 + eta[1] * O21[1];
    O21[1] = eta[0] * O21[1] - eta[1] * tmp1;
    gp[0] = P1[2 * l];
    gp[1] = P1[2 * l + 1];
    gm[0] = P2[2 * l];
    gm[1] = P2[2 * l + 1];
    P1[2 * l] = (O11[0] * gp[0] - O11[1] * gp[1]) + (O12[0] * gm[0] - O12[1] * gm[1]);
    P1[2 * l + 1] = (O11[0] * gp[1] + O11[1] * gp[0]) + (O12[0] * gm[1] + O12[1] * gm[0]);
    P2[2 * l] = (O21[0] * gp[0] - O21[1] * gp[1]) + (O22[0] * gm[0] - O22[1] * gm[1]);
    P2[2 * l + 1] = (O21[0] * gp[1] + O21[1] * gp[0]) + (O22[0] * gm[1] + O22[1] * gm[0]);
  }
}

/* Three-level Bragg step: state 1 (component 0) couples to states 2 and 3
 * (components 1, 2) with Omega_+ and Omega_-; states 2 and 3 share the
 * diagonal V22.  The operation order follows double_bragg.cpp:123-256,
 * including beta . x over all axes (CPoint product), F clipped at 0, and the
 * O32 update that reads the already-updated O23[1] (double_bragg.cpp:233). */
void orc_double_bragg_ad(orc_ctx *c, const orc_laser *L, double F) {
  const double dt = c->dt;
  const double t1 = c->t + 0.5 * dt;
  if (F < 0) F = 0;
  double *P1 = c->psi[0], *P2 = c->psi[1], *P3 = c->psi[2];
  const double *gs = c->gs;
  #pragma omp parallel for schedule(static)
  for (long l = 0; l < c->npts; l++) {
    double x[3];
    orc_get_x(c, l, x);
    double bx = 0;
    for (int a = 0; a < c->dim; a++) bx += L->beta[a] * x[a];
    double tmp1 = P1[2 * l] * P1[2 * l] + P1[2 * l + 1] * P1[2 * l + 1];
    double tmp2 = P2[2 * l] * P2[2 * l] + P2[2 * l + 1] * P2[2 * l + 1];
    double tmp3 = P3[2 * l] * P3[2 * l] + P3[2 * l + 1] * P3[2 * l + 1];
    const double V11 = gs[0] * tmp1 + gs[1] * tmp2 + gs[2] * tmp3 + bx;
    const double V22 = gs[3] * tmp1 + gs[4] * tmp2 + gs[5] * tmp3 - L->DeltaL[1] + bx;
    double dw = L->laser_domh[0] + (L->chirp_rate[0]) * t1;
    const double Op = F * L->Amp[0] * cos(L->laser_k[0] * x[0] - dw * t1 - L->phase[0] / 2);
    dw = L->laser_domh[0] - (L->chirp_rate[0]) * t1;
    const double Om = F * L->Amp[0] * cos(-L->laser_k[0] * x[0] - dw * t1 - L->phase[0] / 2);
    double re1, im1;
    if ((Om == 0.0) && (Op == 0.0)) {
      sincos(-dt * V11, &im1, &re1);
      tmp1 = P1[2 * l];
      P1[2 * l] = tmp1 * re1 - P1[2 * l + 1] * im1;
      P1[2 * l + 1] = tmp1 * im1 + P1[2 * l + 1] * re1;
      sincos(-dt * V22, &im1, &re1);
      tmp1 = P2[2 * l];
      P2[2 * l] = tmp1 * re1 - P2[2 * l + 1] * im1;
      P2[2 * l + 1] = tmp1 * im1 + P2[2 * l + 1] * re1;
      tmp1 = P3[2 * l];
      P3[2 * l] = tmp1 * re1 - P3[2 * l + 1] * im1;
      P3[2 * l + 1] = tmp1 * im1 + P3[2 * l + 1] * re1;
      continue;
    }
    double eta[2], g1[2], g2[2], g3[2];
    double O11[2], O12[2], O13[2], O21[2], O22[2], O23[2], O31[2], O32[2], O33[2];
    sincos(-0.5 * L->laser_dk[0] * x[0], &im1, &re1);
    eta[0] = re1;
    eta[1] = im1;
    tmp1 = sqrt((V11 - V22) * (V11 - V22) + 4.0 * (Op * Op + Om * Om));
    const double E1 = 0.5 * (V11 + V22 + tmp1);
    const double E2 = 0.5 * (V11 + V22 - tmp1);
    sincos(-dt * E1, &im1, &re1);
    tmp1 = 1.0 / fabs((V22 - E1) * (V22 - E1) + Op * Op + Om * Om);
    g1[0] = tmp1 * re1;
    g1[1] = tmp1 * im1;
    sincos(-dt * E2, &im1, &re1);
    tmp1 = 1.0 / fabs((V22 - E2) * (V22 - E2) + Op * Op + Om * Om);
    g2[0] = tmp1 * re1;
    g2[1] = tmp1 * im1;
    sincos(-dt * V22, &im1, &re1);
    tmp1 = 1.0 / fabs(Op * Op + Om * Om);
    g3[0] = tmp1 * re1;
    g3[1] = tmp1 * im1;
    tmp1 = (V22 - E2) * (V22 - E2);
    tmp2 = (V22 - E1) * (V22 - E1);
    O11[0] = tmp1 * g2[0] + tmp2 * g1[0];
    O11[1] = tmp1 * g2[1] + tmp2 * g1[1];
    tmp1 = (V22 - E2) * g2[0] + (V22 - E1) * g1[0];
    tmp2 = (V22 - E2) * g2[1] + (V22 - E1) * g1[1];
    O12[0] = -Op * tmp1;
    O12[1] = -Op * tmp2;
    O13[0] = -Om * tmp1;
    O13[1] = -Om * tmp2;
    O21[0] = O12[0];
    O21[1] = O12[1];
    O31[0] = O13[0];
    O31[1] = O13[1];
    tmp1 = O12[0];
    O12[0] = eta[0] * tmp1 - eta[1] * O12[1];
    O12[1] = eta[1] * tmp1 + eta[0] * O12[1];
    tmp1 = O21[0];
    O21[0] = eta[0] * tmp1 + eta[1] * O21[1];
    O21[1] = eta[0] * O21[1] - eta[1] * tmp1;
    tmp1 = O31[0];
    O31[0] = eta[0] * tmp1 - eta[1] * O31[1];
    O31[1] = eta[1] * tmp1 + eta[0] * O31[1];
    tmp1 = O13[0];
    O13[0] = eta[0] * tmp1 + eta[1] * O13[1];
    O13[1] = eta[0] * O13[1] - eta[1] * tmp1;
    tmp1 = Op * Op;
    tmp2 = Om * Om;
    O22[0] = tmp1 * (g2[0] + g1[0]) + tmp2 * g3[0];
    O22[1] = tmp1 * (g2[1] + g1[1]) + tmp2 * g3[1];
    O33[0] = tmp2 * (g2[0] + g1[0]) + tmp1 * g3[0];
    O33[1] = tmp2 * (g2[1] + g1[1]) + tmp1 * g3[1];
    tmp1 = Om * Op;
    O23[0] = tmp1 * (g1[0] + g2[0] - g3[0]);
    O23[1] = tmp1 * (g1[1] + g2[1] - g3[1]);
    O32[0] = O23[0];
    O32[1] = O23[1];
    tmp1 = O23[0];
    O23[0] = (eta[0] * eta[0] + eta[1] * eta[1]) * tmp1 + 2 * eta[0] * eta[1] * O23[1];
    O23[1] = (eta[0] * eta[0] + eta[1] * eta[1]) * O23[1] - 2 * eta[0] * eta[1] * tmp1;
    tmp1 = O32[0];
    O32[0] = (eta[0] * eta[0] - eta[1] * eta[1]) * tmp1 - 2 * eta[0] * eta[1] * O32[1];
    O32[1] = (eta[0] * eta[0] - eta[1] * eta[1]) * O23[1] + 2 * eta[0] * eta[1] * tmp1;
    g1[0] = P1[2 * l];
    g1[1] = P1[2 * l + 1];
    g2[0] = P2[2 * l];
    g2[1] = P2[2 * l + 1];
    g3[0] = P3[2 * l];
    g3[1] = P3[2 * l + 1];
    P1[2 * l] = (O11[0] * g1[0] - O11[1] * g1[1]) + (O12[0] * g2[0] - O12[1] * g2[1]) + (O13[0] * g3[0] - O13[1] * g3[1]);
    P1[2 * l + 1] = (O11[0] * g1[1] + O11[1] * g1[0]) + (O12[0] * g2[1] + O12[1] * g2[0]) + (O13[0] * g3[1] + O13[1] * g3[0]);
    P2[2 * l] = (O21[0] * g1[0] - O21[1] * g1[1]) + (O22[0] * g2[0] - O22[1] * g2[1]) + (O23[0] * g3[0] - O23[1] * g3[1]);
    P2[2 * l + 1] = (O21[0] * g1[1] + O21[1] * g1[0]) + (O22[0] * g2[1] + O22[1] * g2[0]) + (O23[0] * g3[1] + O23[1] * g3[0]);
    P3[2 * l] = (O31[0] * g1[0] - O31[1] * g1[1]) + (O32[0] * g2[0] - O32[1] * g2[1]) + (O33[0] * g3[0] - O33[1] * g3[1]);
    P3[2 * l + 1] = (O31[0] * g1[1] + O31[1] * g1[0]) + (O32[0] * g2[1] + O32[1] * g2[0]) + (O33[0] * g3[1] + O33[1] * g3[0]);
  }
}

/* ------------------------------------------------- two-species programs */

void orc_set_species2(orc_ctx *c, const orc_laser *L2, double t_start, const double *duration) {
  c->L2 = *L2;
  c->win_t0 = t_start;
  c->win_dur[0] = duration[0];
  c->win_dur[1] = duration[1];
}

/* CRT_Base_IF_2::Do_NL_Step: species 1 = components [0, n/2) with Beta,
 * species 2 = [n/2, n) with Beta_2; phi_i += beta_s x - DeltaL_i as one
 * right-hand side, then *= -dt.  The reference loop is serial. */
void orc_nl_if2_step(orc_ctx *c, const orc_laser *L) {
  const double dt = -c->dt;
  const int n = c->ncomp;
  for (long l = 0; l < c->npts; l++) {
    double phi[ORC_MAXC];
    for (int i = 0; i < n; i++) {
      phi[i] = 0;
      for (int j = 0; j < n; j++) {
        const double *P = c->psi[j];
        phi[i] += c->gs[j + n * i] * (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
      }
      double x[3];
      orc_get_x(c, l, x);
      const double b = (i < n / 2) ? L->beta[0] : c->L2.beta[0];
      phi[i] += b * x[0] - L->DeltaL[i];
      phi[i] *= dt;
    }
    apply_phases(c, l, phi);
  }
}

/* complex products as GCC evaluates std::complex<double> without fused
 * multiply-adds: (a + ib)(c + id) = (ac - bd) + i(ad + bc) */
static inline void zmul(double ar, double ai, double br, double bi, double *r, double *i) {
  *r = ar * br - ai * bi;
  *i = ar * bi + ai * br;
}

/* One species' 2x2 step of bragg_ds.cpp:215-248 on (P, Q) at point l: the
 * eigen-form with complex d0, d1 (imaginary parts zero, so the products
 * reduce to real-times-complex), gamma = e^{-i dt E} / |d^2 + Omega^2| as a
 * complex-by-real division, M01 = ((-Omega) eta) tmp, M10 = ((-Omega)
 * conj(eta)) tmp. */
static void ds_pair(double *P, double *Q, long l, double V11, double V22, double Omega, double er, double ei,
                    double dt) {
  const double tmp1 = sqrt((V11 - V22) * (V11 - V22) + 4.0 * Omega * Omega);
  const double Ep = 0.5 * (V11 + V22 + tmp1);
  const double Em = 0.5 * (V11 + V22 - tmp1);
  const double d0 = V11 - Ep, d1 = V11 - Em;
  double s, co;
  sincos(-dt * Ep, &s, &co);
  const double n0 = fabs(d0 * d0 + Omega * Omega);
  const double g0r = co / n0, g0i = s / n0;
  sincos(-dt * Em, &s, &co);
  const double n1 = fabs(d1 * d1 + Omega * Omega);
  const double g1r = co / n1, g1i = s / n1;
  const double tr = d0 * g0r + d1 * g1r, ti = d0 * g0i + d1 * g1i;
  const double O2 = Omega * Omega;
  const double M00r = O2 * (g0r + g1r), M00i = O2 * (g0i + g1i);
  double M01r, M01i, M10r, M10i;
  zmul(-Omega * er, -Omega * ei, tr, ti, &M01r, &M01i);
  zmul(-Omega * er, -Omega * (-ei), tr, ti, &M10r, &M10i);
  const double q0 = d0 * d0, q1 = d1 * d1;
  const double M11r = q0 * g0r + q1 * g1r, M11i = q0 * g0i + q1 * g1i;
  const double a0r = P[2 * l], a0i = P[2 * l + 1], a1r = Q[2 * l], a1i = Q[2 * l + 1];
  double xr, xi, yr, yi;
  zmul(M00r, M00i, a0r, a0i, &xr, &xi);
  zmul(M01r, M01i, a1r, a1i, &yr, &yi);
  P[2 * l] = xr + yr;
  P[2 * l + 1] = xi + yi;
  zmul(M10r, M10i, a0r, a0i, &xr, &xi);
  zmul(M11r, M11i, a1r, a1i, &yr, &yi);
  Q[2 * l] = xr + yr;
  Q[2 * l + 1] = xi + yi;
}

static void ds_phase(double *P, long l, double phi, double dt) {
  double re1, im1;
  sincos(-phi * dt, &im1, &re1);
  const double tmp1 = P[2 * l];
  P[2 * l] = tmp1 * re1 - P[2 * l + 1] * im1;
  P[2 * l + 1] = tmp1 * im1 + P[2 * l + 1] * re1;
}

/* Bragg_single::Do_Bragg_ad of bragg_ds.  F multiplies both pulse flags
 * (mode1, mode2; 1 reproduces the reference). */
void orc_bragg_ds_ad(orc_ctx *c, const orc_laser *L, double F) {
  const double dt = c->dt;
  const double t1 = c->t + 0.5 * dt;
  const orc_laser *L2 = &c->L2;
  int mode1 = 1, mode2 = 1;
  const double time = t1 - c->win_t0;
  if (time > c->win_dur[0]) mode1 = 0;
  if (time > c->win_dur[1]) mode2 = 0;
  double *P[4] = {c->psi[0], c->psi[1], c->psi[2], c->psi[3]};
  #pragma omp parallel for schedule(static)
  for (long l = 0; l < c->npts; l++) {
    double x[3];
    orc_get_x(c, l, x);
    double phi[4];
    for (int i = 0; i < 4; i++) {
      phi[i] = 0;
      for (int j = 0; j < 4; j++)
        phi[i] += c->gs[j + 4 * i] * (P[j][2 * l] * P[j][2 * l] + P[j][2 * l + 1] * P[j][2 * l + 1]);
      phi[i] += ((i < 2) ? L->beta[0] : L2->beta[0]) * x[0] - L->DeltaL[i];
    }
    const double Omega = (mode1 * F) * L->Amp[0] *
                         cos(L->laser_k[0] * x[0] - (L->laser_domh[0] + L->chirp_rate[0] * t1) * t1 + L->phase[0] / 2);
    const double Omega2 = (mode2 * F) * L2->Amp[0] *
                          cos(L2->laser_k[0] * x[0] - (L2->laser_domh[0] + L2->chirp_rate[0] * t1) * t1 +
                              L2->phase[0] / 2);
    double er, ei;
    if (Omega == 0.0) {
      ds_phase(P[0], l, phi[0], dt);
      ds_phase(P[1], l, phi[1], dt);
    } else {
      sincos(-0.5 * (L->laser_dk[0] * x[0] + L->phase[0]), &ei, &er);
      ds_pair(P[0], P[1], l, phi[0], phi[1], Omega, er, ei, dt);
    }
    if (Omega2 == 0.0) {
      ds_phase(P[2], l, phi[2], dt);
      ds_phase(P[3], l, phi[3], dt);
    } else {
      sincos(-0.5 * (L2->laser_dk[0] * x[0] + L2->phase[0]), &ei, &er);
      ds_pair(P[2], P[3], l, phi[2], phi[3], Omega2, er, ei, dt);
    }
  }
}

/* ------------------------------------------ numerical steps (GSL eigensolver) */

/* Shared tail of Numerical_Bragg / Numerical_Raman: eigen-decompose A, form
 * evec diag(e^{i dt lambda}) evec^H with dt = -header dt, apply it to psi at l. */
typedef struct {
  gsl_matrix_complex *A, *B, *evec;
  gsl_eigen_hermv_workspace *w;
  gsl_vector *eval;
  gsl_vector_complex *P1, *P2;
} orc_num_ws;

static void num_ws_alloc(orc_num_ws *ws, int n) {
  ws->A = gsl_matrix_complex_calloc(n, n);
  ws->B = gsl_matrix_complex_calloc(n, n);
  ws->w = gsl_eigen_hermv_alloc(n);
  ws->eval = gsl_vector_alloc(n);
  ws->P1 = gsl_vector_complex_alloc(n);
  ws->P2 = gsl_vector_complex_alloc(n);
  ws->evec = gsl_matrix_complex_alloc(n, n);
}

static void num_ws_free(orc_num_ws *ws) {
  gsl_matrix_complex_free(ws->A);
  gsl_matrix_complex_free(ws->B);
  gsl_eigen_hermv_free(ws->w);
  gsl_vector_free(ws->eval);
  gsl_vector_complex_free(ws->P1);
  gsl_vector_complex_free(ws->P2);
  gsl_matrix_complex_free(ws->evec);
}

/* diagonal: phi_i = sum_j g_ij |psi_j|^2, then += beta.x - DeltaL_i (CPoint dot
 * product over all axes from 0) */
static void num_diagonal(orc_ctx *c, const orc_laser *L, long l, orc_num_ws *ws, double *phi, double *x) {
  const int n = c->ncomp;
  orc_get_x(c, l, x);
  for (int i = 0; i < n; i++) {
    phi[i] = 0;
    for (int j = 0; j < n; j++) {
      const double *P = c->psi[j];
      phi[i] += c->gs[j + n * i] * (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
    }
    double bx = 0;
    for (int a = 0; a < c->dim; a++) bx += L->beta[a] * x[a];
    phi[i] += bx - L->DeltaL[i];
    gsl_matrix_complex_set(ws->A, i, i, gsl_complex_rect(phi[i], 0));
  }
}

static void num_apply(orc_ctx *c, long l, orc_num_ws *ws) {
  const int n = c->ncomp;
  const double dt = -c->dt;
  gsl_eigen_hermv(ws->A, ws->eval, ws->evec, ws->w);
  for (int i = 0; i < n; i++) {
    double re1, im1;
    sincos(dt * gsl_vector_get(ws->eval, i), &im1, &re1);
    gsl_matrix_complex_set(ws->B, i, i, gsl_complex_rect(re1, im1));
  }
  gsl_blas_zgemm(CblasNoTrans, CblasConjTrans, GSL_COMPLEX_ONE, ws->B, ws->evec, GSL_COMPLEX_ZERO, ws->A);
  gsl_blas_zgemm(CblasNoTrans, CblasNoTrans, GSL_COMPLEX_ONE, ws->evec, ws->A, GSL_COMPLEX_ZERO, ws->B);
  for (int i = 0; i < n; i++) gsl_vector_complex_set(ws->P1, i, gsl_complex_rect(c->psi[i][2 * l], c->psi[i][2 * l + 1]));
  gsl_blas_zgemv(CblasNoTrans, GSL_COMPLEX_ONE, ws->B, ws->P1, GSL_COMPLEX_ZERO, ws->P2);
  for (int i = 0; i < n; i++) {
    c->psi[i][2 * l] = gsl_vector_complex_get(ws->P2, i).dat[0];
    c->psi[i][2 * l + 1] = gsl_vector_complex_get(ws->P2, i).dat[1];
  }
}

/* Numerical_Bragg: state 0 couples to states 1 .. n-1, the second coupling
 * with laser_k[1] = -laser_k[0] and chirp_rate[1] = -chirp_rate[0]; t1 is the
 * header time (no dt/2). */
void orc_numerical_bragg(orc_ctx *c, const orc_laser *L) {
  const int n = c->ncomp;
  const double t1 = c->t;
  const double lk[2] = {L->laser_k[0], -L->laser_k[0]};
  const double cr[2] = {L->chirp_rate[0], -L->chirp_rate[0]};
  orc_num_ws ws;
  num_ws_alloc(&ws, n);
  for (long l = 0; l < c->npts; l++) {
    double phi[ORC_MAXC], x[3];
    gsl_matrix_complex_set_zero(ws.A);
    gsl_matrix_complex_set_zero(ws.B);
    num_diagonal(c, L, l, &ws, phi, x);
    for (int i = 0; i < n - 1; i++) {
      double re1, im1, eta[2];
      sincos(((-L->laser_domh[0] + cr[i] * t1) * t1 + lk[i] * x[0] - 0.5 * L->phase[0]), &im1, &re1);
      eta[0] = L->Amp[0] * re1 / 2 + L->Amp[1] * re1 / 2;
      eta[1] = L->Amp[0] * im1 / 2 - L->Amp[1] * im1 / 2;
      gsl_matrix_complex_set(ws.A, i + 1, 0, gsl_complex_rect(eta[0], eta[1]));
      gsl_matrix_complex_set(ws.A, 0, i + 1, gsl_complex_rect(eta[0], -eta[1]));
    }
    num_apply(c, l, &ws);
  }
  num_ws_free(&ws);
}

/* Numerical_Raman (three states): A_22 += laser_domh, A_02 = Amp0/2 e^{ikx},
 * A_12 = Amp1/2 e^{-ikx}. */
void orc_numerical_raman(orc_ctx *c, const orc_laser *L) {
  orc_num_ws ws;
  num_ws_alloc(&ws, c->ncomp);
  for (long l = 0; l < c->npts; l++) {
    double phi[ORC_MAXC], x[3], re1, im1, eta[2];
    gsl_matrix_complex_set_zero(ws.A);
    gsl_matrix_complex_set_zero(ws.B);
    num_diagonal(c, L, l, &ws, phi, x);
    gsl_matrix_complex_set(ws.A, 2, 2, gsl_complex_rect(phi[2] + L->laser_domh[0], 0));
    sincos((L->laser_k[0] * x[0]), &im1, &re1);
    eta[0] = L->Amp[0] / 2 * re1;
    eta[1] = L->Amp[0] / 2 * im1;
    gsl_matrix_complex_set(ws.A, 0, 2, gsl_complex_rect(eta[0], eta[1]));
    gsl_matrix_complex_set(ws.A, 2, 0, gsl_complex_rect(eta[0], -eta[1]));
    eta[0] = L->Amp[1] / 2 * re1;
    eta[1] = L->Amp[1] / 2 * im1;
    gsl_matrix_complex_set(ws.A, 1, 2, gsl_complex_rect(eta[0], -eta[1]));
    gsl_matrix_complex_set(ws.A, 2, 1, gsl_complex_rect(eta[0], eta[1]));
    num_apply(c, l, &ws);
  }
  num_ws_free(&ws);
}

/* Step kinds: 0 = CRT_Base freeprop, 1 = CRT_Base_IF freeprop, 2 = bragg_ad,
 * 3 = bragg_ad of the three-level double_bragg program, 4 = CRT_Base_IF_2
 * freeprop, 5 = bragg_ad of the two-species bragg_ds program, 6 = the
 * numerical "bragg" step, 7 = the numerical "raman" step (F unused by 6, 7). */
static void nl_dispatch(orc_ctx *c, int kind, const orc_laser *L, double F) {
  if (kind == 0) orc_nl_step(c);
  else if (kind == 1) orc_nl_if_step(c, L);
  else if (kind == 2) orc_bragg_ad(c, L, F);
  else if (kind == 3) orc_double_bragg_ad(c, L, F);
  else if (kind == 4) orc_nl_if2_step(c, L);
  else if (kind == 5) orc_bragg_ds_ad(c, L, F);
  else if (kind == 6) orc_numerical_bragg(c, L);
  else orc_numerical_raman(c, L);
}

/* One outer iteration of run_sequence: half, (V, full)^(Nk-1), V, half.
 * F[j] is the pulse amplitude for the j-th potential step (NULL: 1). */
void orc_block(orc_ctx *c, int nk, int kind, const orc_laser *L, const double *F) {
  orc_ft_step(c, 1);
  for (int j = 2; j <= nk; j++) {
    nl_dispatch(c, kind, L, F ? F[j - 2] : 1.0);
    orc_ft_step(c, 0);
  }
  nl_dispatch(c, kind, L, F ? F[nk - 1] : 1.0);
  orc_ft_step(c, 1);
}

/* ---------------------------------------------------------- observables */

double orc_particle_number(const orc_ctx *c, int comp) {
  const double *P = c->psi[comp];
  double r = 0.0;
  for (long l = 0; l < c->npts; l++) r += (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
  return c->ar * r;
}

void orc_expval_position(const orc_ctx *c, int comp, double *out) {
  const double *P = c->psi[comp];
  double res[3] = {0, 0, 0};
  for (long l = 0; l < c->npts; l++) {
    double x[3];
    orc_get_x(c, l, x);
    const double den = (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
    for (int a = 0; a < c->dim; a++) res[a] += x[a] * den;
  }
  for (int a = 0; a < c->dim; a++) out[a] = c->ar * res[a];
}

void orc_expval_momentum(orc_ctx *c, int comp, double *out) {
  double *P = c->psi[comp];
  double res[3] = {0, 0, 0};
  orc_ft(c, P, -1);
  for (long l = 0; l < c->npts; l++) {
    double k[3];
    orc_get_k(c, l, k);
    const double den = (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
    for (int a = 0; a < c->dim; a++) res[a] += k[a] * den;
  }
  orc_ft(c, P, +1);
  for (int a = 0; a < c->dim; a++) out[a] = c->ar_k * res[a];
}

void orc_setup_momentum(orc_ctx *c, int comp, const double *p) {
  double *P = c->psi[comp];
  for (long l = 0; l < c->npts; l++) {
    double x[3], re, im;
    orc_get_x(c, l, x);
    double dot = 0;
    for (int a = 0; a < c->dim; a++) dot += p[a] * x[a];
    sincos(dot, &im, &re);
    const double re2 = P[2 * l], im2 = P[2 * l + 1];
    P[2 * l] = re2 * re - im2 * im;
    P[2 * l + 1] = re2 * im + im2 * re;
  }
}

/* k0: n points of dim coordinates.  The bin index advances only when a point
 * lies outside a ball, exactly as the reference loop (CRT_Base_IF.h:244-255). */
void orc_rabi_integrals_comp(orc_ctx *c, int comp, const double *k0, int n, double thr, double *out) {
  double *P = c->psi[comp];
  for (int j = 0; j < n; j++) out[j] = 0.0;
  orc_ft(c, P, -1);
  for (long l = 0; l < c->npts; l++) {
    double k1[3];
    orc_get_k(c, l, k1);
    int j = 0;
    for (int m = 0; m < n; m++) {
      double dd = 0;
      for (int a = 0; a < c->dim; a++) {
        const double d = k0[m * c->dim + a] - k1[a];
        dd += d * d;
      }
      if (sqrt(dd) < thr) {
        out[j] += P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1];
        continue;
      }
      j++;
    }
  }
  for (int j = 0; j < n; j++) out[j] = c->ar_k * out[j];
  orc_ft(c, P, +1);
}

void orc_rabi_integrals(orc_ctx *c, const double *k0, int n, double thr, double *out) {
  orc_rabi_integrals_comp(c, 0, k0, n, thr, out);
}

/* -------------------------------------------------------------- sobmin */

/* CSOB_Base::Init (include/CSOB_Base.h:228-248): alpha is Alpha_i[0] on every
 * axis; gs already carries the sqrt(N_i N_j) factor (CSOB_Base.h:177). */
void orc_sob_init(orc_ctx *c, const double *alpha_scalar, double stepsize) {
  c->stepsize = stepsize;
  for (int j = 0; j < c->ncomp; j++) {
    if (!c->op[j]) {
      c->op[j] = (double *)malloc(sizeof(double) * c->npts);
      c->op2[j] = (double *)malloc(sizeof(double) * c->npts);
      c->lap[j] = (double *)calloc((size_t)c->npts * 2, sizeof(double));
      c->sob[j] = (double *)calloc((size_t)c->npts * 2, sizeof(double));
      c->grad[j] = (double *)calloc((size_t)c->npts * 2, sizeof(double));
    }
    for (long i = 0; i < c->npts; i++) {
      double k[3];
      orc_get_k(c, i, k);
      double phi = 0;
      for (int a = 0; a < c->dim; a++) phi += (k[a] * alpha_scalar[j]) * k[a];
      c->op[j][i] = 1.0 / (1.0 + phi);
      c->op2[j][i] = -phi;
    }
  }
}

double *orc_sob_grad(orc_ctx *c, int comp) { return c->grad[comp]; }

static void filter(orc_ctx *c, const double *src, double *dst, const double *op) {
  memcpy(dst, src, sizeof(double) * 2 * c->npts);
  orc_ft(c, dst, -1);
  for (long l = 0; l < c->npts; l++) {
    dst[2 * l] *= op[l];
    dst[2 * l + 1] *= op[l];
  }
  orc_ft(c, dst, +1);
}

static void sob_laplace(orc_ctx *c) {
  for (int i = 0; i < c->ncomp; i++) filter(c, c->psi[i], c->lap[i], c->op2[i]);
}

static double particle_number_raw(const orc_ctx *c, const double *P) {
  double r = 0.0;
  for (long l = 0; l < c->npts; l++) r += (P[2 * l] * P[2 * l] + P[2 * l + 1] * P[2 * l + 1]);
  return c->ar * r;
}

void orc_sob_renormalize(orc_ctx *c) {
  double N[ORC_MAXC];
  for (int i = 0; i < c->ncomp; i++) N[i] = particle_number_raw(c, c->psi[i]);
  for (int i = 0; i < c->ncomp; i++) {
    const double fak = 1.0 / sqrt(N[i]);
    double *P = c->psi[i];
    for (long l = 0; l < c->npts; l++) {
      P[2 * l] *= fak;
      P[2 * l + 1] *= fak;
    }
  }
}

/* One pass of the do-while body of CSOB_Base::run (:433-503).  Returns the
 * residual m_res_tot; N receives the particle numbers it printed. */
double orc_sob_iterate(orc_ctx *c, double *N_out) {
  const int n = c->ncomp;
  for (int i = 0; i < n; i++) filter(c, c->psi[i], c->sob[i], c->op[i]);   /* Compute_Sobolev_Psi */
  sob_laplace(c);                                                          /* Compute_Laplace */
  for (int i = 0; i < n; i++) {                                            /* Compute_Sobolev_Gradient */
    double *G = c->grad[i];
    const double *Psi = c->psi[i], *L = c->lap[i], *pot = c->V[i];
    for (long l = 0; l < c->npts; l++) {
      double NLpot = 0;
      for (int j = 0; j < n; j++)
        NLpot += c->gs[j + i * n] * (c->psi[j][2 * l] * c->psi[j][2 * l] + c->psi[j][2 * l + 1] * c->psi[j][2 * l + 1]);
      const double p = pot ? pot[l] : 0.0;
      G[2 * l] = -L[2 * l] + (p + NLpot) * Psi[2 * l];
      G[2 * l + 1] = -L[2 * l + 1] + (p + NLpot) * Psi[2 * l + 1];
    }
    orc_ft(c, G, -1);
    for (long l = 0; l < c->npts; l++) {
      G[2 * l] *= c->op[i][l];
      G[2 * l + 1] *= c->op[i][l];
    }
    orc_ft(c, G, +1);
  }
  for (int i = 0; i < n; i++) {                                            /* Project_Sobolev_Gradient */
    double *G = c->grad[i];
    const double *Psi = c->psi[i], *S = c->sob[i];
    double tmp1 = 0, tmp2 = 0;
    for (long l = 0; l < c->npts; l++) {
      tmp1 += (Psi[2 * l] * G[2 * l] + Psi[2 * l + 1] * G[2 * l + 1]);
      tmp2 += (Psi[2 * l] * S[2 * l] + Psi[2 * l + 1] * S[2 * l + 1]);
    }
    const double fak = tmp1 / tmp2;
    for (long l = 0; l < c->npts; l++) {
      G[2 * l] -= fak * S[2 * l];
      G[2 * l + 1] -= fak * S[2 * l + 1];
    }
  }
  double res_tot = 0;                                                      /* Compute_res */
  for (int i = 0; i < n; i++) {
    const double *G = c->grad[i];
    double tmp = 0;
    for (long l = 0; l < c->npts; l++) tmp += (G[2 * l] * G[2 * l] + G[2 * l + 1] * G[2 * l + 1]);
    tmp *= c->ar;
    res_tot += tmp * tmp;
  }
  res_tot = sqrt(res_tot);
  int brenorm = 0;
  for (int i = 0; i < n; i++) {
    const double Ni = particle_number_raw(c, c->psi[i]);
    if (N_out) N_out[i] = Ni;
    if (fabs(Ni - 1) > 1e-5) brenorm = 1;
  }
  if (brenorm) orc_sob_renormalize(c);
  for (int i = 0; i < n; i++) {
    double *Psi = c->psi[i];
    const double *G = c->grad[i];
    for (long l = 0; l < c->npts; l++) {
      Psi[2 * l] -= c->stepsize * G[2 * l];
      Psi[2 * l + 1] -= c->stepsize * G[2 * l + 1];
    }
  }
  return res_tot;
}

/* CSOB_Base::run with an iteration cap; returns the iterations taken. */
int orc_sob_run(orc_ctx *c, double epsilon, int max_iter, double *res_out) {
  orc_sob_renormalize(c);
  int it = 0;
  double res;
  do {
    res = orc_sob_iterate(c, NULL);
    it++;
  } while (res > epsilon && it < max_iter);
  if (res_out) *res_out = res;
  return it;
}

/* mu_i = m_ar * sum[-Re(Psi* LapPsi) + (V + sum_j g_ij |Psi_j|^2) |Psi_i|^2]. */
void orc_sob_mu(orc_ctx *c, double *mu) {
  sob_laplace(c);
  const int n = c->ncomp;
  for (int i = 0; i < n; i++) {
    double m = 0;
    const double *Psi = c->psi[i], *L = c->lap[i], *pot = c->V[i];
    for (long l = 0; l < c->npts; l++) {
      double NLpot = 0;
      for (int j = 0; j < n; j++)
        NLpot += c->gs[j + i * n] * (c->psi[j][2 * l] * c->psi[j][2 * l] + c->psi[j][2 * l + 1] * c->psi[j][2 * l + 1]);
      const double p = pot ? pot[l] : 0.0;
      m += -(Psi[2 * l] * L[2 * l] + Psi[2 * l + 1] * L[2 * l + 1]) +
           (p + NLpot) * (Psi[2 * l] * Psi[2 * l] + Psi[2 * l + 1] * Psi[2 * l + 1]);
    }
    mu[i] = c->ar * m;
  }
}

/* Raw transform access for the FFT known-answer tests. */
void orc_fft_raw(orc_ctx *c, double *data, int isign) {
  orc_fft_execute(isign < 0 ? c->fwd : c->bwd, data);
}
void orc_set_threads(int n) {
  orc_fft_set_threads(n);
  if (n > 0) omp_set_num_threads(n);
}

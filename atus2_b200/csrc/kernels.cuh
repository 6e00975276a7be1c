// kernels.cuh -- split-step kernels of the ATUS-2 engine (sm_100a).
//
// Fields live in HBM as one contiguous array per component, row-major with x
// slowest (the .bin layout): complex128 in FP64 mode, complex64 in mixed mode.
//
// pass_kernel  one HBM read and one HBM write of a tile of pencils along one
//              axis: [transform] -> point-wise operator -> [transform].  Used
//              as  FFT_a -> kinetic phase -> IFFT_a   (k-space half-step) and
//              IFFT_a -> potential/Bragg step -> FFT_a (real-space half-step),
//              so each Strang step of a 2D grid is two passes over the fields.
// block1d_kernel  1D grids: a whole Strang block (Nk steps) with the field
//              resident in shared memory.
// nl_kernel    the potential step alone (Do_NL_Step / Do_Bragg_ad).
// reduce_*     deterministic two-level FP64 reductions.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "fft_device.cuh"

namespace atus {

constexpr int MAXC = 4;
constexpr int TWN = 16384;  // twiddle table length (largest supported pencil)

// Per-CTA tile budget in complex elements and threads per CTA.
template <typename R> struct Tile;
// MINB: CTAs per SM the register budget is sized for (two tiles resident per
// SM, so one CTA's loads overlap the other's transforms).
template <> struct Tile<double> { static constexpr int E = 2048; static constexpr int NT = 128; static constexpr int MINB = 3; };
template <> struct Tile<float> { static constexpr int E = 4096; static constexpr int NT = 256; static constexpr int MINB = 3; };

constexpr int BLOCK1D_NT = 256;  // threads of the resident 1D Strang-block kernel

enum { T_NONE = 0, T_FWD = -1, T_INV = 1 };
enum { OP_NONE = 0, OP_KIN = 1, OP_NL = 2, OP_FILT = 3 };
enum { FILT_SOBOLEV = 0, FILT_LAPLACE = 1 };
// step kinds: CRT_Base freeprop, CRT_Base_IF freeprop, bragg_ad, the
// three-level bragg_ad (double_bragg), CRT_Base_IF_2 freeprop (two species),
// the two-species bragg_ad (bragg_ds), and the numerical n-state "bragg" and
// three-state "raman" steps of CRT_Base_IF
enum { K_NL = 0, K_NL_IF = 1, K_BRAGG = 2, K_DBRAGG = 3, K_NL_IF2 = 4, K_BRAGG_DS = 5, K_NUM_BRAGG = 6, K_RAMAN = 7 };
// modes of the register-staged pass kernel (pass2.cuh)
// M2_KIN_RABI: M2_KIN that also sums |psi^(k)|^2 over the Rabi balls of the
// requested components while every axis is in k-space (the last kinetic pass
// of a block); a separate instantiation, so M2_KIN keeps its registers.
enum { M2_FWD = 0, M2_INV = 1, M2_KIN = 2, M2_NL = 3, M2_KIN_RABI = 4 };

struct LaserD {
  double beta0, DeltaL[MAXC], Amp0, laser_k0, laser_dk0, laser_domh0, phase0, chirp_rate0, chirp;
  double Amp1;  // second amplitude (Amp_1 entry 1), used by the numerical steps
};

// Potential-step parameters (by value).
struct NLArgs {
  int kind;                 // K_NL / K_NL_IF / K_BRAGG
  int ncomp;
  double mdt;               // -dt
  double dt;
  double gs[MAXC * MAXC];   // gs[i * MAXC + j] = g_ij (GS_(i+1) entry j)
  const double *V[MAXC];    // nullptr: no potential
  LaserD L;
  double t1;                // header t + dt/2
  double F;                 // pulse amplitude
  double dx0;               // grid step of axis 0
  int shift0;               // n0 / 2
  int stable;               // FP64 Bragg step in the eigenvalue-free form (1) or the reference's (0)
  // three-level Bragg step: beta . x over every axis (grid steps, centres and
  // log2 lengths of axes 1 and 2 to recover y and z from the grid index)
  double beta1, beta2, dx1, dx2;
  int shift1, shift2, lg1, lg2;
  // second species of the two-species programs (beta0, Amp0, laser_k0,
  // laser_dk0, laser_domh0, phase0, chirp_rate0 used) and its pulse factor
  LaserD L2;
  double F2;
  double th;  // header time at the potential step (the numerical "bragg" step's t1)
};

struct Geo {
  int lg[3];                // log2 of n0, n1, n2 (unused axes: 0)
  int64_t npts;
};

struct PassArgs {
  void *psi[MAXC];
  int nc;                   // components in the tile (NL) or 1 (per-component passes)
  int per_comp;             // 1: blockIdx.y selects the component
  int64_t sa;               // pencil stride in elements
  int64_t inner_tiles;      // strided: tiles per outer block; contiguous: unused
  int64_t npencils;         // contiguous: number of pencils
  int64_t ntiles;           // tiles per component
  int ncomp_grid;           // components walked by per-component passes
  int t1, op, t2;
  const double2 *kt[MAXC][3];  // kinetic phase factors per component and axis (FP64)
  double s_f, s_b;          // forward / backward transform scales (cft_*d::scale)
  const void *tw;           // twiddles exp(-2 pi i m / TWN)
  Geo g;
  NLArgs nl;
  int x_along;              // 1 when the pencil runs along axis 0 (x varies inside a pencil)
  int axis;                 // axis the pencils run along
  // OP_FILT: real k-space filter of CSOB_Base (include/CSOB_Base.h:228-248):
  // 1/(1 + alpha k^2) or -alpha k^2, times the transform scale.
  int filt_mode;
  double filt_alpha, filt_scale;
  double dk[3];
  int n[3];
  // M2_KIN_RABI: balls k0[c * rabi_n + m] (m < rabi_n) of component
  // rabi_comp[c] (c < rabi_ncomp), radius rabi_thr; per-CTA sums of the
  // unscaled |psi^|^2 to rabi_partial[blockIdx.x * 8 + q]
  int rabi_ncomp, rabi_n;
  int rabi_comp[2];
  double rabi_thr;
  double rabi_k0[8][3];
  double *rabi_partial;
  int *err;  // device error word (bounded waits that ran out set bits)
  long wait_limit;       // try_wait rounds before a TMA tile counts as lost
  int drop_copies;       // issue no tile copies, so every wait runs out (error-path tests; 0)
};

__device__ __forceinline__ void idx3(const Geo &g, int64_t l, int &ix, int &iy, int &iz) {
  ix = (int)(l >> (g.lg[1] + g.lg[2]));
  iy = (int)((l >> g.lg[2]) & ((1 << g.lg[1]) - 1));
  iz = (int)(l & ((1 << g.lg[2]) - 1));
}

// ------------------------------------------------------------ phase helpers
// a - 2 pi rint(a / 2 pi), Cody-Waite with 2 pi = P1 + P2 (+P3), P1 with 32
// significant bits so q*P1 is exact for |q| < 2^20.
__device__ __forceinline__ double reduce_2pi(double a) {
  const double P1 = 6.2831853069365025, P2 = 2.430840202602477e-10, P3 = 1.40862394607328e-26;
  const double q = rint(a * 0.15915494309189535);
  double r = fma(-q, P1, a);
  r = fma(-q, P2, r);
  return fma(-q, P3, r);
}

// sin and cos of an FP64 argument.  The phases of a time step are small
// (|dt V| << 1 in practice), so |x| <= 1/32 takes the Taylor polynomials
//   sin x = x (1 - x^2/3! + x^4/5! - x^6/7! + x^8/9!)
//   cos x = 1 - x^2/2! + x^4/4! - x^6/6! + x^8/8! - x^10/10!
// whose truncation errors (x^11/11!, x^12/12!) are below 2^-70 there, in
// Horner form on x^2; larger arguments call sincos().
__device__ __forceinline__ void sincos_step(double x, double *s, double *c) {
  if (fabs(x) <= 0.03125) {
    // Taylor series to x^7 (sin) and x^8 (cos): the first omitted terms,
    // x^9/9! and x^10/10!, are below 2.5e-18 x and 2.5e-22 for |x| <= 1/32
    const double x2 = x * x;
    double ps = fma(x2, -1.0 / 5040.0, 1.0 / 120.0);
    ps = fma(ps, x2, -1.0 / 6.0);
    *s = fma(ps * x2, x, x);
    double pc = fma(x2, 1.0 / 40320.0, -1.0 / 720.0);
    pc = fma(pc, x2, 1.0 / 24.0);
    pc = fma(pc, x2, -0.5);
    *c = fma(pc, x2, 1.0);
  } else {
    sincos(x, s, c);
  }
}

// Element of MAXC-entry arrays by a runtime index without local memory.
template <typename T> __device__ __forceinline__ T pick(const T (&a)[MAXC], int i) {
  T r = a[0];
  if (i == 1) r = a[1];
  if (i == 2) r = a[2];
  if (i == 3) r = a[3];
  return r;
}

template <typename R> __device__ __forceinline__ double2 to_d(cplx<R> v) { return make_double2((double)v.x, (double)v.y); }
template <typename R> __device__ __forceinline__ cplx<R> from_d(double2 v) { return mk<R>((R)v.x, (R)v.y); }

// Unit phase factor e^{i phi} in FP64.  Mixed precision: FP64 argument
// reduced modulo 2 pi, sincosf, then renormalised in FP64 so that |e| = 1 to
// FP64 accuracy (a fixed modulus error would drift the norm every step).
template <typename R> __device__ __forceinline__ double2 expi(double phi);
template <> __device__ __forceinline__ double2 expi<double>(double phi) {
  double s, c;
  sincos_step(phi, &s, &c);
  return make_double2(c, s);
}
template <> __device__ __forceinline__ double2 expi<float>(double phi) {
  if (fabs(phi) <= 0.03125) {  // the usual phase of one time step: FP64 Taylor, |e| = 1 to FP64
    double sd, cd;
    sincos_step(phi, &sd, &cd);
    return make_double2(cd, sd);
  }
  float s, c;
  sincosf((float)reduce_2pi(phi), &s, &c);
  const double cd = c, sd = s;
  const double inv = rsqrt(cd * cd + sd * sd);
  return make_double2(cd * inv, sd * inv);
}

// ------------------------------------------------------------ three-level Bragg step
// Bragg_double::Do_Double_Bragg_ad (source/interferometry/src/double_bragg.cpp:
// 123-256) at grid index l: state 1 (component 0) couples to states 2 and 3
// with Omega_+ = F Amp cos(k x - (domh + rate t1) t1 - phase/2) and Omega_- =
// F Amp cos(-k x - (domh - rate t1) t1 - phase/2); states 2 and 3 share V22;
// V includes beta . x over all axes.  The reference's operation order,
// including its O32 update that reads the already-updated O23 imaginary part
// (double_bragg.cpp:233).  FP64 arithmetic for both field precisions.
template <typename R>
__device__ __forceinline__ void dbragg_point(const NLArgs &a, cplx<R> *v, int64_t l, double x0) {
  double bx = a.L.beta0 * x0;
  if (a.lg1 > 0) {
    const int iy = (int)((l >> a.lg2) & ((1 << a.lg1) - 1));
    bx += a.beta1 * ((double)(iy - a.shift1) * a.dx1);
  }
  if (a.lg2 > 0) {
    const int iz = (int)(l & ((1 << a.lg2) - 1));
    bx += a.beta2 * ((double)(iz - a.shift2) * a.dx2);
  }
  const double2 p1 = to_d<R>(v[0]), p2 = to_d<R>(v[1]), p3 = to_d<R>(v[2]);
  double tmp1 = p1.x * p1.x + p1.y * p1.y;
  double tmp2 = p2.x * p2.x + p2.y * p2.y;
  const double tmp3 = p3.x * p3.x + p3.y * p3.y;
  const double *gs = a.gs;  // padded rows: g_ij at i * MAXC + j
  const double V11 = gs[0] * tmp1 + gs[1] * tmp2 + gs[2] * tmp3 + bx;
  const double V22 = gs[MAXC] * tmp1 + gs[MAXC + 1] * tmp2 + gs[MAXC + 2] * tmp3 - a.L.DeltaL[1] + bx;
  const double t1 = a.t1, dt = a.dt;
  const double F = a.F < 0 ? 0.0 : a.F;
  double dw = a.L.laser_domh0 + a.L.chirp_rate0 * t1;
  const double Op = F * a.L.Amp0 * cos(a.L.laser_k0 * x0 - dw * t1 - a.L.phase0 / 2);
  dw = a.L.laser_domh0 - a.L.chirp_rate0 * t1;
  const double Om = F * a.L.Amp0 * cos(-a.L.laser_k0 * x0 - dw * t1 - a.L.phase0 / 2);
  double re1, im1;
  if (Om == 0.0 && Op == 0.0) {
    sincos_step(-dt * V11, &im1, &re1);
    v[0] = from_d<R>(cmul(p1, make_double2(re1, im1)));
    sincos_step(-dt * V22, &im1, &re1);
    v[1] = from_d<R>(cmul(p2, make_double2(re1, im1)));
    v[2] = from_d<R>(cmul(p3, make_double2(re1, im1)));
    return;
  }
  double e0, e1;
  sincos(-0.5 * a.L.laser_dk0 * x0, &e1, &e0);
  const double OO = Op * Op + Om * Om;
  tmp1 = sqrt((V11 - V22) * (V11 - V22) + 4.0 * OO);
  const double E1 = 0.5 * (V11 + V22 + tmp1);
  const double E2 = 0.5 * (V11 + V22 - tmp1);
  double2 g1, g2, g3;
  sincos_step(-dt * E1, &im1, &re1);
  tmp1 = 1.0 / fabs((V22 - E1) * (V22 - E1) + Op * Op + Om * Om);
  g1 = make_double2(tmp1 * re1, tmp1 * im1);
  sincos_step(-dt * E2, &im1, &re1);
  tmp1 = 1.0 / fabs((V22 - E2) * (V22 - E2) + Op * Op + Om * Om);
  g2 = make_double2(tmp1 * re1, tmp1 * im1);
  sincos_step(-dt * V22, &im1, &re1);
  tmp1 = 1.0 / fabs(OO);
  g3 = make_double2(tmp1 * re1, tmp1 * im1);
  tmp1 = (V22 - E2) * (V22 - E2);
  tmp2 = (V22 - E1) * (V22 - E1);
  const double2 O11 = make_double2(tmp1 * g2.x + tmp2 * g1.x, tmp1 * g2.y + tmp2 * g1.y);
  tmp1 = (V22 - E2) * g2.x + (V22 - E1) * g1.x;
  tmp2 = (V22 - E2) * g2.y + (V22 - E1) * g1.y;
  const double2 A12 = make_double2(-Op * tmp1, -Op * tmp2);  // O12 = O21 before eta
  const double2 A13 = make_double2(-Om * tmp1, -Om * tmp2);  // O13 = O31 before eta
  const double2 O12 = make_double2(e0 * A12.x - e1 * A12.y, e1 * A12.x + e0 * A12.y);
  const double2 O21 = make_double2(e0 * A12.x + e1 * A12.y, e0 * A12.y - e1 * A12.x);
  const double2 O31 = make_double2(e0 * A13.x - e1 * A13.y, e1 * A13.x + e0 * A13.y);
  const double2 O13 = make_double2(e0 * A13.x + e1 * A13.y, e0 * A13.y - e1 * A13.x);
  tmp1 = Op * Op;
  tmp2 = Om * Om;
  const double2 O22 = make_double2(tmp1 * (g2.x + g1.x) + tmp2 * g3.x, tmp1 * (g2.y + g1.y) + tmp2 * g3.y);
  const double2 O33 = make_double2(tmp2 * (g2.x + g1.x) + tmp1 * g3.x, tmp2 * (g2.y + g1.y) + tmp1 * g3.y);
  tmp1 = Om * Op;
  const double2 A23 = make_double2(tmp1 * (g1.x + g2.x - g3.x), tmp1 * (g1.y + g2.y - g3.y));
  const double ep = e0 * e0 + e1 * e1, em = e0 * e0 - e1 * e1, e2 = 2 * e0 * e1;
  const double2 O23 = make_double2(ep * A23.x + e2 * A23.y, ep * A23.y - e2 * A23.x);
  const double2 O32 = make_double2(em * A23.x - e2 * A23.y, em * O23.y + e2 * A23.x);
  v[0] = from_d<R>(cadd(cadd(cmul(O11, p1), cmul(O12, p2)), cmul(O13, p3)));
  v[1] = from_d<R>(cadd(cadd(cmul(O21, p1), cmul(O22, p2)), cmul(O23, p3)));
  v[2] = from_d<R>(cadd(cadd(cmul(O31, p1), cmul(O32, p2)), cmul(O33, p3)));
}

// ------------------------------------------------------------ two-level exponential
// exp(-i dt [[V11, Omega eta], [Omega conj(eta), V22]]) applied to (p1, p2).
// FP64 and not `stable`: the reference's eigenvalue form (bragg.cpp:226-302,
// bragg_ds.cpp:215-248): E+- = (V11 + V22 +- sqrt((V11 - V22)^2 + 4 Omega^2))/2,
// gamma+- = e^{-i dt E+-} / |(V11 - E+-)^2 + Omega^2|, pure phases when
// Omega == 0.  Otherwise the eigenvalue-free form
//   U = e^{-i dt m} [cos(r dt) I - i sin(r dt)/r [[d, W], [W, -d]]],
// m = (V11+V22)/2, d = (V11-V22)/2, W = Omega, r = sqrt(d^2 + W^2), built in
// FP64 from unit (cos, sin) pairs, so it is unitary to FP64 accuracy for every
// Omega (the eigenvalue form divides by (V11 - E)^2 + Omega^2, which loses
// unitarity once Omega is below the spacing of V and divides by zero once
// Omega^2 underflows).
template <typename R>
__device__ __forceinline__ void bragg_pair(int stable, double dt, double V11, double V22, double Omega, double eta_c,
                                           double eta_s, cplx<R> &q1, cplx<R> &q2) {
  if constexpr (sizeof(R) == 8) {
    if (!stable) {
      double re1, im1;
      if (Omega == 0.0) {
        sincos_step(-dt * V11, &im1, &re1);
        q1 = cmul(q1, make_double2(re1, im1));
        sincos_step(-dt * V22, &im1, &re1);
        q2 = cmul(q2, make_double2(re1, im1));
        return;
      }
      double tmp1 = sqrt((V11 - V22) * (V11 - V22) + 4.0 * Omega * Omega);
      const double Ep = 0.5 * (V11 + V22 + tmp1);
      const double Em = 0.5 * (V11 + V22 - tmp1);
      double2 gp, gm;
      // the reference's 1 / |(V11 - E+-)^2 + Omega^2| (sums of squares, so
      // |.| is the identity) from one division: 1/A = B/(AB), 1/B = A/(AB)
      const double Ap = (V11 - Ep) * (V11 - Ep) + Omega * Omega;
      const double Am = (V11 - Em) * (V11 - Em) + Omega * Omega;
      const double inv = 1.0 / (Ap * Am);
      sincos_step(-dt * Ep, &im1, &re1);
      tmp1 = Am * inv;
      gp = make_double2(tmp1 * re1, tmp1 * im1);
      sincos_step(-dt * Em, &im1, &re1);
      tmp1 = Ap * inv;
      gm = make_double2(tmp1 * re1, tmp1 * im1);
      const double O2 = Omega * Omega;
      const double2 O11 = make_double2(O2 * (gp.x + gm.x), O2 * (gp.y + gm.y));
      const double a1 = V11 - Ep, a2 = V11 - Em;
      const double2 O22 = make_double2(a1 * a1 * gp.x + a2 * a2 * gm.x, a1 * a1 * gp.y + a2 * a2 * gm.y);
      const double2 Os = make_double2(-Omega * (a1 * gp.x + a2 * gm.x), -Omega * (a1 * gp.y + a2 * gm.y));
      const double2 eta = make_double2(eta_c, eta_s);
      const double2 O12 = cmul(Os, eta);   // eta * O12
      const double2 O21 = cmulc(Os, eta);  // conj(eta) * O21
      const double2 p1 = q1, p2 = q2;
      q1 = cadd(cmul(O11, p1), cmul(O12, p2));
      q2 = cadd(cmul(O21, p1), cmul(O22, p2));
      return;
    }
  }
  const double m = 0.5 * (V11 + V22), d = 0.5 * (V11 - V22);
  const double r = sqrt(d * d + Omega * Omega);
  const double2 e = expi<R>(-dt * m);   // e^{-i dt m}
  const double2 rr = expi<R>(dt * r);   // (cos r dt, sin r dt)
  // sin(r dt) / r: Taylor series of sinc (truncation below 2^-72 for r dt <= 1/32)
  const double xr = dt * r;
  double sor;
  if (xr <= 0.03125) {
    const double x2 = xr * xr;
    double p = fma(x2, 1.0 / 362880.0, -1.0 / 5040.0);
    p = fma(p, x2, 1.0 / 120.0);
    p = fma(p, x2, -1.0 / 6.0);
    sor = dt * fma(p, x2, 1.0);
  } else {
    sor = rr.y / r;
  }
  const double fd = sor * d, fw = sor * Omega;
  // U11 = e(cos - i fd), U22 = e(cos + i fd), Uoff = e(-i fw)
  const double2 U11 = cmul(e, make_double2(rr.x, -fd));
  const double2 U22 = cmul(e, make_double2(rr.x, fd));
  const double2 Uo = cmul(e, make_double2(0.0, -fw));
  const double2 et = make_double2(eta_c, eta_s);
  const double2 U12 = cmul(Uo, et), U21 = cmulc(Uo, et);
  const double2 p1 = to_d<R>(q1), p2 = to_d<R>(q2);
  q1 = from_d<R>(cadd(cmul(U11, p1), cmul(U12, p2)));
  q2 = from_d<R>(cadd(cmul(U21, p1), cmul(U22, p2)));
}

// ------------------------------------------------------------ two-species Bragg step
// Bragg_single::Do_Bragg_ad of the two-species program (source/interferometry/
// src/bragg_ds.cpp:111-322) at grid index l: components (0, 1) are species 1,
// (2, 3) species 2; V_i = sum_j g_ij |psi_j|^2 + (beta_s x - DeltaL_i) with
// beta_s of the component's species (x along axis 0 only); species s couples
// with Omega_s = F_s Amp_s cos(k_s x - (domh_s + rate_s t1) t1 + phase_s/2),
// eta_s = e^{-i (dk_s x + phase_s)/2}.  F_s is 0 outside the species' pulse
// window (bragg_ds.cpp:117-127), set on the host.
template <typename R>
__device__ __forceinline__ void bragg_ds_point(const NLArgs &a, cplx<R> *v, double x0) {
  double rho[MAXC];
  #pragma unroll
  for (int j = 0; j < MAXC; j++) rho[j] = (double)v[j].x * (double)v[j].x + (double)v[j].y * (double)v[j].y;
  double phi[MAXC];
  #pragma unroll
  for (int i = 0; i < MAXC; i++) {
    double p = a.gs[i * MAXC] * rho[0];
    #pragma unroll
    for (int j = 1; j < MAXC; j++) p += a.gs[i * MAXC + j] * rho[j];
    phi[i] = p + (((i < 2) ? a.L.beta0 : a.L2.beta0) * x0 - a.L.DeltaL[i]);
  }
  const double t1 = a.t1, dt = a.dt;
  #pragma unroll
  for (int s = 0; s < 2; s++) {
    const LaserD &L = s ? a.L2 : a.L;
    const double Omega = (s ? a.F2 : a.F) * L.Amp0 *
                         cos(L.laser_k0 * x0 - (L.laser_domh0 + L.chirp_rate0 * t1) * t1 + L.phase0 / 2);
    double es, ec;
    sincos(-0.5 * (L.laser_dk0 * x0 + L.phase0), &es, &ec);
    bragg_pair<R>(a.stable, dt, phi[2 * s], phi[2 * s + 1], Omega, ec, es, v[2 * s], v[2 * s + 1]);
  }
}

// ------------------------------------------------------------ numerical n-state steps
// psi <- exp(-i h A) psi for a Hermitian 3x3 matrix A (n = 2: the third row
// and column are zero and so is psi[2]).  The reference diagonalises A with
// GSL's gsl_eigen_hermv and forms V diag(e^{-i h lambda}) V^H psi
// (include/CRT_Base_IF.h:471-497, 581-607); here the same exponential comes
// from its Taylor series on the vector: the mean of the diagonal is taken out
// as a scalar phase, the rest is split into s substeps with
// h ||A||_inf / s <= 1/4 (||.||_inf bounded by |Re| + |Im| row sums), and each
// substep sums terms (-i h A / s)^k psi / k! until a term falls below 2^-60
// of the sum (k <= 18; the truncation error at k = 18 is below 1e-22).  No
// eigenvalues, so degenerate or nearly degenerate spectra need no care.
__device__ __forceinline__ void herm_expm_apply(double2 (&A)[3][3], int n, double h, double2 (&p)[3]) {
  double mu = 0.0;
  #pragma unroll
  for (int i = 0; i < 3; i++)
    if (i < n) mu += A[i][i].x;
  mu /= n;
  #pragma unroll
  for (int i = 0; i < 3; i++)
    if (i < n) A[i][i].x -= mu;
  double nu = 0.0;
  #pragma unroll
  for (int i = 0; i < 3; i++) {
    double r = 0.0;
    #pragma unroll
    for (int j = 0; j < 3; j++) r += fabs(A[i][j].x) + fabs(A[i][j].y);
    nu = fmax(nu, r);
  }
  nu *= h;
  int steps = 1;
  if (nu > 0.25) steps = (int)fmin(ceil(4.0 * nu), 1048576.0);
  const double hs = h / steps;
  // M = -i hs A
  double2 M[3][3];
  #pragma unroll
  for (int i = 0; i < 3; i++)
    #pragma unroll
    for (int j = 0; j < 3; j++) M[i][j] = make_double2(hs * A[i][j].y, -hs * A[i][j].x);
  constexpr double INVK[19] = {0.0,      1.0,       1.0 / 2,  1.0 / 3,  1.0 / 4,  1.0 / 5,  1.0 / 6,
                               1.0 / 7,  1.0 / 8,   1.0 / 9,  1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13,
                               1.0 / 14, 1.0 / 15,  1.0 / 16, 1.0 / 17, 1.0 / 18};
  for (int st = 0; st < steps; st++) {
    double2 y[3] = {p[0], p[1], p[2]}, t[3] = {p[0], p[1], p[2]};
    #pragma unroll 1
    for (int k = 1; k <= 18; k++) {
      double2 u[3];
      #pragma unroll
      for (int i = 0; i < 3; i++) {
        double2 acc = cmul(M[i][0], t[0]);
        acc = cadd(acc, cmul(M[i][1], t[1]));
        acc = cadd(acc, cmul(M[i][2], t[2]));
        u[i] = make_double2(acc.x * INVK[k], acc.y * INVK[k]);
      }
      double tn = 0.0, yn = 0.0;
      #pragma unroll
      for (int i = 0; i < 3; i++) {
        t[i] = u[i];
        y[i] = cadd(y[i], u[i]);
        tn += fabs(u[i].x) + fabs(u[i].y);
        yn += fabs(y[i].x) + fabs(y[i].y);
      }
      if (tn <= 0x1p-60 * yn) break;
    }
    p[0] = y[0];
    p[1] = y[1];
    p[2] = y[2];
  }
  double sn, cs;
  sincos_step(-h * mu, &sn, &cs);
  const double2 e = make_double2(cs, sn);
  #pragma unroll
  for (int i = 0; i < 3; i++) p[i] = cmul(p[i], e);
}

// beta . x over every axis at grid index l (x0 given; y and z from the index).
__device__ __forceinline__ double beta_dot_x(const NLArgs &a, int64_t l, double x0) {
  double bx = a.L.beta0 * x0;
  if (a.lg1 > 0) {
    const int iy = (int)((l >> a.lg2) & ((1 << a.lg1) - 1));
    bx += a.beta1 * ((double)(iy - a.shift1) * a.dx1);
  }
  if (a.lg2 > 0) {
    const int iz = (int)(l & ((1 << a.lg2) - 1));
    bx += a.beta2 * ((double)(iz - a.shift2) * a.dx2);
  }
  return bx;
}

// The numerical steps of CRT_Base_IF at grid index l (n = ncomp components):
// diagonal V_i = sum_j g_ij |psi_j|^2 + (beta . x - DeltaL_i);
//  "bragg" (Numerical_Bragg, include/CRT_Base_IF.h:426-526): state 0 couples
//   to state i+1 with eta_i = (Amp0 + Amp1)/2 cos(a_i) + i (Amp0 - Amp1)/2
//   sin(a_i), a_i = (-domh + rate_i t) t + k_i x - phase/2, k_1 = -k_0,
//   rate_1 = -rate_0, t the header time;
//  "raman" (Numerical_Raman, :533-632): V_2 + domh, A_02 = Amp0/2 e^{i k x},
//   A_12 = Amp1/2 e^{-i k x}.
// Then psi <- exp(-i dt A) psi in FP64 for both field precisions.
// Not inlined: the pass kernels that carry it keep their register budget for
// the common steps.
template <typename R, int TC>
__device__ __noinline__ void num_point(const NLArgs &a, cplx<R> *v, int64_t l, double x0) {
  constexpr int NC = TC < 3 ? TC : 3;
  const int n = a.ncomp;
  const double bx = beta_dot_x(a, l, x0);
  double2 p[3];
  double rho[3];
  #pragma unroll
  for (int j = 0; j < 3; j++) {
    p[j] = (j < NC && j < n) ? to_d<R>(v[j]) : make_double2(0.0, 0.0);
    rho[j] = p[j].x * p[j].x + p[j].y * p[j].y;
  }
  double2 A[3][3];
  #pragma unroll
  for (int i = 0; i < 3; i++)
    #pragma unroll
    for (int j = 0; j < 3; j++) A[i][j] = make_double2(0.0, 0.0);
  #pragma unroll
  for (int i = 0; i < NC; i++) {
    if (i >= n) break;
    double phi = 0.0;
    #pragma unroll
    for (int j = 0; j < NC; j++)
      if (j < n) phi += a.gs[i * MAXC + j] * rho[j];
    A[i][i].x = phi + (bx - a.L.DeltaL[i]);
  }
  if (a.kind == K_RAMAN) {
    if constexpr (NC >= 3) {
      A[2][2].x += a.L.laser_domh0;
      double sn, cs;
      sincos(a.L.laser_k0 * x0, &sn, &cs);
      const double h0 = a.L.Amp0 / 2, h1 = a.L.Amp1 / 2;
      A[0][2] = make_double2(h0 * cs, h0 * sn);
      A[2][0] = make_double2(h0 * cs, -h0 * sn);
      A[1][2] = make_double2(h1 * cs, -h1 * sn);
      A[2][1] = make_double2(h1 * cs, h1 * sn);
    }
  } else {
    const double t1 = a.th;
    #pragma unroll
    for (int i = 0; i + 1 < NC; i++) {
      if (i + 1 >= n) break;
      const double k = i == 0 ? a.L.laser_k0 : -a.L.laser_k0;
      const double rate = i == 0 ? a.L.chirp_rate0 : -a.L.chirp_rate0;
      double sn, cs;
      sincos((-a.L.laser_domh0 + rate * t1) * t1 + k * x0 - 0.5 * a.L.phase0, &sn, &cs);
      const double er = a.L.Amp0 * cs / 2 + a.L.Amp1 * cs / 2, ei = a.L.Amp0 * sn / 2 - a.L.Amp1 * sn / 2;
      A[i + 1][0] = make_double2(er, ei);
      A[0][i + 1] = make_double2(er, -ei);
    }
  }
  herm_expm_apply(A, n, a.dt, p);
  #pragma unroll
  for (int j = 0; j < NC; j++)
    if (j < n) v[j] = from_d<R>(p[j]);
}


// ------------------------------------------------------------ potential step
// Point-wise potential step on the ncomp values v[] at grid index l.
// FP64: the reference's formulas (include/CRT_Base.h:410-439,
// CRT_Base_IF.h:392-418, bragg.cpp:210-302).  Mixed: FP64 phase arguments,
// FP32 field arithmetic, and the eigenvalue-free form of the 2x2 exponential.
// TC: the number of components the calling kernel holds (ncomp <= TC); step
// kinds that need more components are compiled out.  PREV (one component):
// the caller has loaded the potential at l into vpre (0 without a potential).
template <typename R, int TC = MAXC, bool PREV = false>
__device__ __forceinline__ void nl_point(const NLArgs &a, cplx<R> *v, int64_t l, double x0, double Omega,
                                         double eta_c, double eta_s, double vpre = 0.0) {
  static_assert(!PREV || TC == 1, "a pre-loaded potential serves one component");
  if constexpr (TC >= 3) {
    if (a.kind == K_DBRAGG) {
      dbragg_point<R>(a, v, l, x0);
      return;
    }
  }
  if constexpr (TC >= 4) {
    if (a.kind == K_BRAGG_DS) {
      bragg_ds_point<R>(a, v, x0);
      return;
    }
  }
  if constexpr (TC >= 2) {
    if (a.kind == K_NUM_BRAGG || a.kind == K_RAMAN) {
      // the out-of-line step gets a copy: were the caller's array handed to
      // it, its address would escape and the array would live in local
      // memory on every path
      cplx<R> w[TC];
      #pragma unroll
      for (int c = 0; c < TC; c++) w[c] = v[c];
      num_point<R, TC>(a, w, l, x0);
      #pragma unroll
      for (int c = 0; c < TC; c++) v[c] = w[c];
      return;
    }
  }
  const int n = a.ncomp;
  double rho[TC];
  #pragma unroll
  for (int j = 0; j < TC; j++)
    if (j < n) rho[j] = (double)v[j].x * (double)v[j].x + (double)v[j].y * (double)v[j].y;
  if (TC < 2 || a.kind != K_BRAGG) {
    #pragma unroll
    for (int i = 0; i < TC; i++) {
      if (i >= n) break;
      double phi;
      if (a.kind == K_NL) {
        if constexpr (PREV) phi = vpre;
        else phi = a.V[i] ? a.V[i][l] : 0.0;
        #pragma unroll
        for (int j = 0; j < TC; j++)
          if (j < n) phi += a.gs[i * MAXC + j] * rho[j];
      } else {
        phi = 0.0;
        #pragma unroll
        for (int j = 0; j < TC; j++)
          if (j < n) phi += a.gs[i * MAXC + j] * rho[j];
        // CRT_Base_IF_2 (two species): beta of the component's species
        const double b = (a.kind == K_NL_IF2 && 2 * i >= n) ? a.L2.beta0 : a.L.beta0;
        phi += b * x0 - a.L.DeltaL[i];
      }
      phi *= a.mdt;
      const double2 e = expi<R>(phi);
      v[i] = from_d<R>(cmul(to_d<R>(v[i]), e));
    }
    return;
  }
  if constexpr (TC >= 2) {
    // Bragg 2x2 (components 0 and 1)
    const double V11 = a.gs[0] * rho[0] + a.gs[1] * rho[1] + a.L.beta0 * x0;
    const double V22 = a.gs[MAXC] * rho[0] + a.gs[MAXC + 1] * rho[1] - a.L.DeltaL[1] + a.L.beta0 * x0;
    bragg_pair<R>(a.stable, a.dt, V11, V22, Omega, eta_c, eta_s, v[0], v[1]);
  }
}

// Omega(x0) and eta(x0) of the Bragg step (bragg.cpp:224, 243).
__device__ __forceinline__ void bragg_coupling(const NLArgs &a, double x0, double &Omega, double &ec, double &es) {
  const double t1 = a.t1;
  Omega = a.F * a.L.Amp0 *
          cos(a.L.laser_k0 * x0 - (a.L.laser_domh0 + a.L.chirp * t1 + a.L.chirp_rate0 * t1) * t1 + a.L.phase0 / 2);
  sincos(-0.5 * (a.L.laser_dk0 * x0), &es, &ec);
}

// ------------------------------------------------------------ kinetic step
template <typename C>
__device__ __forceinline__ C kin_phase(const C *kx, const C *ky, const C *kz, int ix, int iy, int iz) {
  return cmul(cmul(__ldg(&kx[ix]), __ldg(&ky[iy])), __ldg(&kz[iz]));
}

// ------------------------------------------------------------ pass kernel
// Asynchronous global -> shared copies (cp.async): a tile's loads are issued
// without registers and complete while the previous tile is transformed.
__device__ __forceinline__ void cp_async(void *smem, const void *gmem, double2) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async(void *smem, const void *gmem, float2) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::); }

template <typename R, int N, int TC>
struct PassCfg {
  static constexpr int NT = Tile<R>::NT;
  static constexpr int B0 = Tile<R>::E / (N * TC);
  static constexpr int B1 = B0 > 0 ? B0 : 1;
  static constexpr int B = B1 < 256 ? B1 : 256;  // pencils per tile
  static constexpr int NP = Pad<N>::NP;
  static constexpr int TILE = TC * B * NP;       // complex values per buffer
  // two buffers (prefetch of the next work item) when they fit, else one
  static constexpr int NBUF = (2 * sizeof(cplx<R>) * (size_t)TILE + 3 * 8 * B <= 227 * 1024) ? 2 : 1;
  static constexpr size_t smem = NBUF * sizeof(cplx<R>) * (size_t)TILE;
};

struct TileGeo {
  int64_t base0;    // grid index of element 0 of pencil 0
  int64_t pstride;  // distance between the tile's pencils
  int nb;           // pencils of the tile inside the grid
  int comp0;        // first component
};

template <int B, int N>
__device__ __forceinline__ TileGeo tile_geo(const PassArgs &a, int64_t w) {
  TileGeo g;
  int64_t t = w;
  g.comp0 = 0;
  if (a.per_comp) {
    g.comp0 = (int)(w / a.ntiles);
    t = w % a.ntiles;
  }
  if (a.sa > 1) {
    const int64_t o = t / a.inner_tiles;
    const int64_t r0 = (t % a.inner_tiles) * B;
    g.base0 = o * (int64_t)N * a.sa + r0;
    g.pstride = 1;
    g.nb = (int)((a.sa - r0) < B ? (a.sa - r0) : B);
  } else {
    const int64_t p0 = t * B;
    g.base0 = p0 * N;
    g.pstride = N;
    g.nb = (int)((a.npencils - p0) < B ? (a.npencils - p0) : B);
  }
  return g;
}

// Persistent pass kernel: each CTA walks work items (tile, component) with a
// stride of the grid size, double buffered -- the cp.async loads of item w+1
// fly while item w is transformed and stored.
template <typename R, int N, int TC>
__global__ void __launch_bounds__(Tile<R>::NT, Tile<R>::MINB) pass_kernel(PassArgs a) {
  using C = cplx<R>;
  using Cfg = PassCfg<R, N, TC>;
  constexpr int B = Cfg::B, NT = Cfg::NT, NP = Cfg::NP, TILE = Cfg::TILE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *const sbase = reinterpret_cast<C *>(smem_raw);
  __shared__ double s_om[B], s_ec[B], s_es[B];
  static_assert((B * N) % NT == 0, "tile must be a multiple of the CTA size");
  constexpr int LPT = B * N / NT;
  const int64_t W = a.per_comp ? a.ntiles * a.ncomp_grid : a.ntiles;
  const typename TwTab<R>::type *tw = (const typename TwTab<R>::type *)a.tw;

  auto issue = [&](int64_t w, C *s) {
    const TileGeo g = tile_geo<B, N>(a, w);
    const int nc = a.per_comp ? 1 : a.nc;
    #pragma unroll
    for (int c = 0; c < TC; c++) {
      const C *src = (const C *)pick(a.psi, g.comp0 + c);
      #pragma unroll
      for (int k = 0; k < LPT; k++) {
        const int r = threadIdx.x + k * NT;
        int b, i;
        if (a.sa > 1) { b = r % B; i = r / B; } else { i = r % N; b = r / N; }
        C *dst = &s[c * B * NP + Pad<N>::idx(b, i)];
        if (c < nc && b < g.nb) cp_async(dst, &src[g.base0 + b * g.pstride + (int64_t)i * a.sa], C{});
        else *dst = mk<R>(0, 0);
      }
    }
  };

  int64_t w = blockIdx.x;
  int buf = 0;
  if (Cfg::NBUF == 2) {
    if (w < W) issue(w, sbase);
    cp_commit();
  }
  for (; w < W; w += gridDim.x) {
    C *s = sbase + buf * TILE;
    if (Cfg::NBUF == 2) {
      const int64_t wn = w + gridDim.x;
      if (wn < W) issue(wn, sbase + (buf ^ 1) * TILE);
      cp_commit();
      cp_wait_prev();
    } else {
      issue(w, s);
      cp_commit();
      asm volatile("cp.async.wait_all;\n" ::);
    }
    __syncthreads();

    const TileGeo g = tile_geo<B, N>(a, w);
    const int nc = a.per_comp ? 1 : a.nc;
    const int64_t base0 = g.base0, pstride = g.pstride;
    const int nb = g.nb, comp0 = g.comp0;
    if (a.t1 == T_FWD) fft_tile<R, N, TC * B, NT, -1, TWN>(s, tw);
    else if (a.t1 == T_INV) fft_tile<R, N, TC * B, NT, +1, TWN>(s, tw);

    if (a.op == OP_KIN) {
      // psi^ <- ((psi^ s_f) K) s_b with K = Kx Ky Kz in FP64: the two scales of
      // the reference's ft(-1) / ft(+1) as separate products (no folded,
      // once-rounded constant that would bias every step the same way)
      const double2 *kx = a.kt[0][0], *ky = a.kt[0][1], *kz = a.kt[0][2];
      #pragma unroll
      for (int c = 1; c < MAXC; c++)
        if (comp0 == c) { kx = a.kt[c][0]; ky = a.kt[c][1]; kz = a.kt[c][2]; }
      #pragma unroll 4
      for (int e = threadIdx.x; e < B * N; e += NT) {
        const int b = e / N, i = e % N;
        if (b < nb) {
          const int64_t l = base0 + b * pstride + (int64_t)i * a.sa;
          int ix, iy, iz;
          idx3(a.g, l, ix, iy, iz);
          const double2 k = kin_phase(kx, ky, kz, ix, iy, iz);
          const int si = Pad<N>::idx(b, i);
          double2 v = to_d<R>(s[si]);
          v.x *= a.s_f;
          v.y *= a.s_f;
          v = cmul(v, k);
          v.x *= a.s_b;
          v.y *= a.s_b;
          s[si] = from_d<R>(v);
        }
      }
      __syncthreads();
    } else if (a.op == OP_FILT) {
      for (int e = threadIdx.x; e < B * N; e += NT) {
        const int b = e / N, i = e % N;
        if (b < nb) {
          const int64_t l = base0 + b * pstride + (int64_t)i * a.sa;
          int ijk[3];
          idx3(a.g, l, ijk[0], ijk[1], ijk[2]);
          double phi = 0;
          #pragma unroll
          for (int ax = 0; ax < 3; ax++) {
            const int t = (ijk[ax] + a.n[ax] / 2) % a.n[ax];
            const double k = a.dk[ax] * (double)(t - a.n[ax] / 2);
            phi += (k * a.filt_alpha) * k;
          }
          const double f = (a.filt_mode == FILT_SOBOLEV ? 1.0 / (1.0 + phi) : -phi) * a.filt_scale;
          const int si = Pad<N>::idx(b, i);
          C v = s[si];
          v.x = (R)((double)v.x * f);
          v.y = (R)((double)v.y * f);
          s[si] = v;
        }
      }
      __syncthreads();
    } else if (a.op == OP_NL) {
      const bool bragg = (a.nl.kind == K_BRAGG);
      if (bragg && !a.x_along) {
        for (int b = threadIdx.x; b < B; b += NT) {
          double om = 0, ec = 1, es = 0;
          if (b < nb) {
            int ix, iy, iz;
            idx3(a.g, base0 + b * pstride, ix, iy, iz);
            bragg_coupling(a.nl, (double)(ix - a.nl.shift0) * a.nl.dx0, om, ec, es);
          }
          s_om[b] = om; s_ec[b] = ec; s_es[b] = es;
        }
        __syncthreads();
      }
      #pragma unroll 2
      for (int e = threadIdx.x; e < B * N; e += NT) {
        const int b = e / N, i = e % N;
        if (b < nb) {
          const int64_t l = base0 + b * pstride + (int64_t)i * a.sa;
          int ix, iy, iz;
          idx3(a.g, l, ix, iy, iz);
          const double x0 = (double)(ix - a.nl.shift0) * a.nl.dx0;
          double om = 0, ec = 1, es = 0;
          if (bragg) {
            if (a.x_along) bragg_coupling(a.nl, x0, om, ec, es);
            else { om = s_om[b]; ec = s_ec[b]; es = s_es[b]; }
          }
          C v[MAXC];
          #pragma unroll
          for (int c = 0; c < TC; c++) v[c] = s[c * B * NP + Pad<N>::idx(b, i)];
          nl_point<R, TC>(a.nl, v, l, x0, om, ec, es);
          #pragma unroll
          for (int c = 0; c < TC; c++) s[c * B * NP + Pad<N>::idx(b, i)] = v[c];
        }
      }
      __syncthreads();
    }

    if (a.t2 == T_FWD) fft_tile<R, N, TC * B, NT, -1, TWN>(s, tw);
    else if (a.t2 == T_INV) fft_tile<R, N, TC * B, NT, +1, TWN>(s, tw);

    #pragma unroll
    for (int c = 0; c < TC; c++) {
      if (c < nc) {
        C *dst = (C *)pick(a.psi, comp0 + c);
        #pragma unroll
        for (int k = 0; k < LPT; k++) {
          const int r = threadIdx.x + k * NT;
          int b, i;
          if (a.sa > 1) { b = r % B; i = r / B; } else { i = r % N; b = r / N; }
          if (b < nb) dst[base0 + b * pstride + (int64_t)i * a.sa] = s[c * B * NP + Pad<N>::idx(b, i)];
        }
      }
    }
    __syncthreads();  // the buffer is refilled two items later
    if (Cfg::NBUF == 2) buf ^= 1;
  }
  asm volatile("cp.async.wait_all;\n" ::);
}

// ------------------------------------------------------------ 1D Strang block
struct Block1DArgs {
  void *psi[MAXC];
  const double2 *kh[MAXC], *kf[MAXC];  // half / full kinetic phase factors (FP64)
  double s_f, s_b;                     // forward / backward transform scales
  const void *tw;
  NLArgs nl;
  int nk;
  double t0;                        // header time at block start
  const double *F;                  // per potential step, or nullptr
};

template <typename R, int N, int TC>
__device__ __forceinline__ void kin_1d(cplx<R> *s, const double2 *const (&tab)[TC], int nc, double s_f, double s_b) {
  constexpr int NT = BLOCK1D_NT, NP = Pad<N>::NP;
  #pragma unroll
  for (int c = 0; c < TC; c++) {
    if (c < nc) {
      for (int i = threadIdx.x; i < N; i += NT) {
        const int si = c * NP + Pad<N>::idx(0, i);
        double2 v = to_d<R>(s[si]);
        v.x *= s_f;
        v.y *= s_f;
        v = cmul(v, __ldg(&tab[c][i]));
        v.x *= s_b;
        v.y *= s_b;
        s[si] = from_d<R>(v);
      }
    }
  }
  __syncthreads();
}

template <typename R, int N, int TC>
__global__ void __launch_bounds__(BLOCK1D_NT) block1d_kernel(Block1DArgs a) {
  using C = cplx<R>;
  constexpr int NT = BLOCK1D_NT, NP = Pad<N>::NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  const int nc = a.nl.ncomp;
  const typename TwTab<R>::type *tw = (const typename TwTab<R>::type *)a.tw;
  C *fld[TC];
  const double2 *kh[TC], *kf[TC];
  #pragma unroll
  for (int c = 0; c < TC; c++) {
    fld[c] = (C *)a.psi[c];
    kh[c] = a.kh[c];
    kf[c] = a.kf[c];
  }
  #pragma unroll
  for (int c = 0; c < TC; c++)
    for (int i = threadIdx.x; i < N; i += NT) s[c * NP + Pad<N>::idx(0, i)] = (c < nc) ? fld[c][i] : mk<R>(0, 0);
  __syncthreads();
  double t = a.t0;
  const double dt = a.nl.dt;
  // half kinetic step
  fft_tile<R, N, TC, NT, -1, TWN>(s, tw);
  kin_1d<R, N, TC>(s, kh, nc, a.s_f, a.s_b);
  fft_tile<R, N, TC, NT, +1, TWN>(s, tw);
  t += 0.5 * dt;
  // the step parameters in shared memory (thread 0 sets the step's time and
  // pulse amplitude): a per-thread copy of the ~0.5 KB block sat in local memory
  __shared__ NLArgs s_nl;
  const NLArgs &nl = s_nl;
  if (threadIdx.x == 0) s_nl = a.nl;
  for (int j = 0; j < a.nk; j++) {
    if (threadIdx.x == 0) {
      s_nl.t1 = t + 0.5 * dt;
      s_nl.F = a.F ? a.F[j] : 1.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < N; i += NT) {
      const double x0 = (double)(i - nl.shift0) * nl.dx0;
      double om = 0, ec = 1, es = 0;
      if (nl.kind == K_BRAGG) bragg_coupling(nl, x0, om, ec, es);
      C v[MAXC];
      #pragma unroll
      for (int c = 0; c < TC; c++) v[c] = s[c * NP + Pad<N>::idx(0, i)];
      nl_point<R, TC>(nl, v, i, x0, om, ec, es);
      #pragma unroll
      for (int c = 0; c < TC; c++) s[c * NP + Pad<N>::idx(0, i)] = v[c];
    }
    __syncthreads();
    const bool last = (j == a.nk - 1);
    fft_tile<R, N, TC, NT, -1, TWN>(s, tw);
    if (last) kin_1d<R, N, TC>(s, kh, nc, a.s_f, a.s_b);
    else kin_1d<R, N, TC>(s, kf, nc, a.s_f, a.s_b);
    fft_tile<R, N, TC, NT, +1, TWN>(s, tw);
    t += last ? 0.5 * dt : dt;
  }
  #pragma unroll
  for (int c = 0; c < TC; c++)
    if (c < nc)
      for (int i = threadIdx.x; i < N; i += NT) fld[c][i] = s[c * NP + Pad<N>::idx(0, i)];
}

// ------------------------------------------------------------ point-wise kernels
struct NLKArgs {
  void *psi[MAXC];
  NLArgs nl;
  Geo g;
};

template <typename R>
__global__ void nl_kernel(NLKArgs a) {
  using C = cplx<R>;
  const int n = a.nl.ncomp;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < a.g.npts;
       l += (int64_t)gridDim.x * blockDim.x) {
    int ix, iy, iz;
    idx3(a.g, l, ix, iy, iz);
    const double x0 = (double)(ix - a.nl.shift0) * a.nl.dx0;
    double om = 0, ec = 1, es = 0;
    if (a.nl.kind == K_BRAGG) bragg_coupling(a.nl, x0, om, ec, es);
    C v[MAXC];
    #pragma unroll
    for (int c = 0; c < MAXC; c++)
      if (c < n) v[c] = ((C *)a.psi[c])[l];
    nl_point<R>(a.nl, v, l, x0, om, ec, es);
    #pragma unroll
    for (int c = 0; c < MAXC; c++)
      if (c < n) ((C *)a.psi[c])[l] = v[c];
  }
}

// psi *= e^{i p.x}  (Setup_Momentum)
template <typename R>
__global__ void momentum_kernel(void *psi, Geo g, double p0, double p1, double p2, double dx0, double dx1,
                                double dx2, int s0, int s1, int s2) {
  using C = cplx<R>;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < g.npts; l += (int64_t)gridDim.x * blockDim.x) {
    int ix, iy, iz;
    idx3(g, l, ix, iy, iz);
    const double dot = p0 * ((double)(ix - s0) * dx0) + p1 * ((double)(iy - s1) * dx1) + p2 * ((double)(iz - s2) * dx2);
    C *P = (C *)psi;
    P[l] = from_d<R>(cmul(to_d<R>(P[l]), expi<R>(dot)));
  }
}

// FP64 <-> field precision conversions (mixed mode upload / download).
template <typename R>
__global__ void convert_in_kernel(void *dst, const double2 *src, int64_t n) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x)
    ((cplx<R> *)dst)[l] = mk<R>((R)src[l].x, (R)src[l].y);
}
template <typename R>
__global__ void convert_out_kernel(double2 *dst, const void *src, int64_t n) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    const cplx<R> v = ((const cplx<R> *)src)[l];
    dst[l] = make_double2((double)v.x, (double)v.y);
  }
}

// ------------------------------------------------------------ Sobolev helpers
// G = -Lap psi_i + (V_i + sum_j g_ij |psi_j|^2) psi_i   (CSOB_Base.h:317-326)
struct SobArgs {
  const double2 *psi[MAXC];
  const double2 *lap;
  const double *V;
  double2 *grad;
  double2 *copy;  // when set, also receives psi[comp]
  int comp, ncomp;
  double gs[MAXC * MAXC];
  int64_t npts;
};

// ------------------------------------------------------------ reductions
// Quantities per mode (all FP64 accumulations, fixed order per thread, fixed
// tree per block, partials summed in block order by reduce_final).
enum { RED_NORM = 0, RED_POS = 1, RED_MOM = 2, RED_RABI = 3, RED_DOT2 = 4, RED_MU = 5, RED_PROJ = 6, RED_SOBG = 7 };
constexpr int RED_MAXQ = 8;
constexpr int RED_BLOCKS = 592;  // 4 x 148 SMs
constexpr int RED_THREADS = 256;

struct RedArgs {
  int mode;
  int nq;
  const void *a, *b, *c;   // field operands
  const double *V;
  Geo g;
  int dim;
  double d[3], dk[3];
  int n[3], shift[3];
  double k0[8][3];         // Rabi centres
  double thr;
  // mu
  const void *psi_all[MAXC];
  int ncomp, comp;
  double gs[MAXC * MAXC];
  // projection: w <- w - (fq[0] / fq[1]) c, then |w|^2 (FP64 fields)
  double2 *w;
  const double *fq;
};

template <typename R>
__device__ __forceinline__ void red_point(const RedArgs &a, int64_t l, double *q) {
  using C = cplx<R>;
  if (a.mode == RED_SOBG) {
    // w = S(W psi) becomes the Sobolev gradient S(-Lap psi + W psi) =
    // S(W psi) + psi - S psi (S = 1/(1 + alpha k^2), so S alpha k^2 = 1 - S),
    // then Re<psi, G>, Re<psi, S psi>, <psi, psi>
    const double2 p = ((const double2 *)a.a)[l], ps = ((const double2 *)a.c)[l];
    double2 g = a.w[l];
    g.x += p.x - ps.x;
    g.y += p.y - ps.y;
    a.w[l] = g;
    q[0] += p.x * g.x + p.y * g.y;
    q[1] += p.x * ps.x + p.y * ps.y;
    q[2] += p.x * p.x + p.y * p.y;
    return;
  }
  if (a.mode == RED_PROJ) {  // Project_Sobolev_Gradient and the norm of the result in one pass
    const double fak = a.fq[0] / a.fq[1];
    double2 v = a.w[l];
    const double2 u = ((const double2 *)a.c)[l];
    v.x -= fak * u.x;
    v.y -= fak * u.y;
    a.w[l] = v;
    q[0] += v.x * v.x + v.y * v.y;
    return;
  }
  const C v = ((const C *)a.a)[l];
  const double den = (double)v.x * (double)v.x + (double)v.y * (double)v.y;
  if (a.mode == RED_NORM) { q[0] += den; return; }
  int ijk[3];
  idx3(a.g, l, ijk[0], ijk[1], ijk[2]);
  if (a.mode == RED_POS) {
    for (int ax = 0; ax < a.dim; ax++) q[ax] += ((double)(ijk[ax] - a.shift[ax]) * a.d[ax]) * den;
    return;
  }
  double k[3];
  for (int ax = 0; ax < a.dim; ax++) {
    const int t = (ijk[ax] + a.shift[ax]) % a.n[ax];
    k[ax] = a.dk[ax] * (double)(t - a.shift[ax]);
  }
  if (a.mode == RED_MOM) {
    for (int ax = 0; ax < a.dim; ax++) q[ax] += k[ax] * den;
    return;
  }
  if (a.mode == RED_RABI) {
    int j = 0;
    for (int m = 0; m < a.nq; m++) {
      double dd = 0;
      for (int ax = 0; ax < a.dim; ax++) {
        const double d = a.k0[m][ax] - k[ax];
        dd += d * d;
      }
      if (sqrt(dd) < a.thr) { q[j] += den; continue; }
      j++;
    }
    return;
  }
  if (a.mode == RED_DOT2) {  // Re<a,b>, Re<a,c> (and <a,a> when nq is 3)
    const C b = ((const C *)a.b)[l];
    q[0] += (double)v.x * (double)b.x + (double)v.y * (double)b.y;
    if (a.c) {
      const C c = ((const C *)a.c)[l];
      q[1] += (double)v.x * (double)c.x + (double)v.y * (double)c.y;
    }
    if (a.nq > 2) q[2] += den;
    return;
  }
  if (a.mode == RED_MU) {  // a = psi_i, b = Lap psi_i
    const C lp = ((const C *)a.b)[l];
    double nl = 0;
    #pragma unroll
    for (int j = 0; j < MAXC; j++) {
      if (j < a.ncomp) {
        const C pj = ((const C *)a.psi_all[j])[l];
        nl += a.gs[a.comp * MAXC + j] * ((double)pj.x * (double)pj.x + (double)pj.y * (double)pj.y);
      }
    }
    const double pot = a.V ? a.V[l] : 0.0;
    q[0] += -((double)v.x * (double)lp.x + (double)v.y * (double)lp.y) + (pot + nl) * den;
  }
}

template <typename R>
__global__ void __launch_bounds__(RED_THREADS) reduce_kernel(RedArgs a, double *partial) {
  double q[RED_MAXQ];
  #pragma unroll
  for (int i = 0; i < RED_MAXQ; i++) q[i] = 0;
  for (int64_t l = blockIdx.x * (int64_t)RED_THREADS + threadIdx.x; l < a.g.npts; l += (int64_t)gridDim.x * RED_THREADS)
    red_point<R>(a, l, q);
  __shared__ double sh[RED_THREADS];
  for (int i = 0; i < a.nq; i++) {
    sh[threadIdx.x] = q[i];
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x * RED_MAXQ + i] = sh[0];
    __syncthreads();
  }
}


}  // namespace atus

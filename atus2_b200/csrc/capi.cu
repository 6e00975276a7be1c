// capi.cu -- host side of libatus_gpu.so: context, planning of the fused
// passes, and the extern "C" entry points declared in include/atus_gpu.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/atus_gpu.h"
#include "ctx.h"
#include "launch.h"
#include "kernels_host.cuh"

using namespace atus;

static int ilog2(int64_t v) {
  int l = 0;
  while ((int64_t(1) << l) < v) l++;
  return l;
}

// ------------------------------------------------------------------ tables
// exp(-2 pi i m / TWN) in long double, rounded once; quarter turns exact.
template <typename R> static std::vector<cplx<R>> twiddles() {
  std::vector<cplx<R>> t(TWN);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < TWN; m++) {
    long double c, s;
    if (m == 0) { c = 1; s = 0; }
    else if (4 * m == TWN) { c = 0; s = 1; }
    else if (2 * m == TWN) { c = -1; s = 0; }
    else if (4 * m == 3 * TWN) { c = 0; s = -1; }
    else {
      const long double th = two_pi * (long double)m / (long double)TWN;
      c = cosl(th);
      s = sinl(th);
    }
    t[m].x = (R)c;
    t[m].y = (R)(-s);
  }
  return t;
}

// Scale factors of cft_Nd::scale (cft_1d.cpp:191-201, cft_2d.cpp:449-459,
// cft_3d.cpp:627-637): forward uses dx.., backward dk..
static double scale_fak(int dim, const double *s) {
  if (dim == 1) return s[0] / sqrt(2.0 * M_PI);
  if (dim == 2) return 0.5 * s[0] * s[1] / M_PI;
  return s[0] * s[1] * s[2] / pow(2 * M_PI, 1.5);
}

static int64_t wrapped(int64_t i, int64_t n) { return ((i + n / 2) % n) - n / 2; }

// Scale of one forward+inverse round trip, folded into the kinetic phase.  For
// headers written as gen_psi_0 / Get_Header write them (dx = L/N, dk = 2 pi/L)
// the product is exactly 1/N_total, a power of two; it is used exactly then,
// so the folded scale adds no rounding (what matters for complex64 fields).
static double round_trip_scale(const atus_ctx *ctx) {
  const double s = scale_fak(ctx->dim, ctx->d) * scale_fak(ctx->dim, ctx->dk);
  const double exact = 1.0 / (double)ctx->npts;
  return (fabs(s - exact) <= 1e-12 * exact) ? exact : s;
}

// Kinetic phase factors per axis, in FP64 for both precisions, evaluated with
// the reference's own double arithmetic (include/CRT_Base.h:257-271):
// phi = (-dt) * ((k alpha) k), factor (cos(phi/2), sin(phi/2)) for the half
// step and (cos phi, sin phi) for the full one.  In 1D this is the reference's
// table bit for bit; in 2D/3D the factor of a k-point is the product of the
// axis factors.  The transform scales stay separate (applied in the kernel).
static int build_kinetic(atus_ctx *ctx) {
  for (int hf = 0; hf < 2; hf++) {
    for (int c = 0; c < ctx->ncomp; c++) {
      for (int ax = 0; ax < 3; ax++) {
        const int64_t n = ctx->n[ax];
        std::vector<double2> tab(n);
        for (int64_t i = 0; i < n; i++) {
          double phi = 0.0;
          if (ax < ctx->dim) {
            const double k = ctx->dk[ax] * (double)wrapped(i, n);
            phi = (-ctx->dt) * ((k * ctx->alpha[c][ax]) * k);
          }
          tab[i].x = (hf == 0) ? cos(0.5 * phi) : cos(phi);
          tab[i].y = (hf == 0) ? sin(0.5 * phi) : sin(phi);
        }
        if (!ctx->kt[hf][c][ax]) CK(cudaMalloc(&ctx->kt[hf][c][ax], sizeof(double2) * n));
        CK(cudaMemcpyAsync(ctx->kt[hf][c][ax], tab.data(), sizeof(double2) * n, cudaMemcpyHostToDevice, ctx->stream));
      }
    }
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return ATUS_OK;
}

// ------------------------------------------------------------------ launch helpers
static NLArgs nl_args(const atus_ctx *ctx, int kind, double t1, double F) {
  NLArgs a;
  memset(&a, 0, sizeof(a));
  a.kind = kind;
  a.ncomp = ctx->ncomp;
  a.mdt = -ctx->dt;
  a.dt = ctx->dt;
  for (int i = 0; i < MAXC * MAXC; i++) a.gs[i] = ctx->gs[i];
  for (int c = 0; c < MAXC; c++) a.V[c] = (c < ctx->ncomp) ? ctx->V[c] : nullptr;
  a.L.beta0 = ctx->laser.beta[0];
  for (int c = 0; c < MAXC; c++) a.L.DeltaL[c] = ctx->laser.DeltaL[c];
  a.L.Amp0 = ctx->laser.Amp[0];
  a.L.Amp1 = ctx->laser.Amp[1];
  a.L.laser_k0 = ctx->laser.laser_k[0];
  a.L.laser_dk0 = ctx->laser.laser_dk[0];
  a.L.laser_domh0 = ctx->laser.laser_domh[0];
  a.L.phase0 = ctx->laser.phase[0];
  a.L.chirp_rate0 = ctx->laser.chirp_rate[0];
  a.L.chirp = ctx->laser.chirp;
  a.t1 = t1;
  a.F = F;
  a.dx0 = ctx->d[0];
  a.shift0 = (int)(ctx->n[0] / 2);
  a.stable = ctx->bragg_stable;
  a.beta1 = ctx->laser.beta[1];
  a.beta2 = ctx->laser.beta[2];
  a.dx1 = ctx->d[1];
  a.dx2 = ctx->d[2];
  a.shift1 = (int)(ctx->n[1] / 2);
  a.shift2 = (int)(ctx->n[2] / 2);
  a.lg1 = ctx->lg[1];
  a.lg2 = ctx->lg[2];
  a.L2.beta0 = ctx->laser2.beta[0];
  a.L2.Amp0 = ctx->laser2.Amp[0];
  a.L2.laser_k0 = ctx->laser2.laser_k[0];
  a.L2.laser_dk0 = ctx->laser2.laser_dk[0];
  a.L2.laser_domh0 = ctx->laser2.laser_domh[0];
  a.L2.phase0 = ctx->laser2.phase[0];
  a.L2.chirp_rate0 = ctx->laser2.chirp_rate[0];
  a.F2 = F;
  a.th = ctx->t;
  if (kind == K_BRAGG_DS) {
    // mode1 / mode2 of bragg_ds.cpp:117-127: time = t1 - seq.time
    const double time = t1 - ctx->win_t0;
    if (time > ctx->win_dur[0]) a.F = 0.0;
    if (time > ctx->win_dur[1]) a.F2 = 0.0;
  }
  return a;
}

static int tc_for(int ncomp) { return ncomp <= 1 ? 1 : (ncomp <= 2 ? 2 : 4); }

// The register-staged kernel where it has an instantiation (pencils of 32..256
// points, the pass shapes of the split-step schedule), else the tile kernel.
static int dispatch_pass(atus_ctx *ctx, PassArgs &a, int axis, int tc) {
  const bool dbl = (ctx->prec == ATUS_PREC_FP64);
  if (ctx->use_pass2) {
    const bool strided = axis < ctx->dim - 1;
    int r = ATUS_E_UNSUPPORTED;
    if (a.op == OP_NONE && a.t2 == T_NONE && (a.t1 == T_FWD || a.t1 == T_INV)) {
      const int mode = (a.t1 == T_FWD) ? M2_FWD : M2_INV;
      r = dbl ? launch_pass2_d_t(ctx, a, axis, mode, strided) : launch_pass2_f_t(ctx, a, axis, mode, strided);
    } else if ((a.op == OP_KIN || a.op == OP_FILT) && a.t1 == T_FWD && a.t2 == T_INV && strided) {
      r = dbl ? launch_pass2_d_k(ctx, a, axis) : launch_pass2_f_k(ctx, a, axis);
    } else if (a.op == OP_NL && a.t1 == T_INV && a.t2 == T_FWD && !strided && tc <= 2) {
      r = dbl ? launch_pass2_d_nl(ctx, a, axis, tc) : launch_pass2_f_nl(ctx, a, axis, tc);
    }
    if (r != ATUS_E_UNSUPPORTED) return r;
  }
  if (dbl) {
    if (tc == 1) return launch_pass_d1(ctx, a, axis);
    if (tc == 2) return launch_pass_d2(ctx, a, axis);
    return launch_pass_d4(ctx, a, axis);
  }
  if (tc == 1) return launch_pass_f1(ctx, a, axis);
  if (tc == 2) return launch_pass_f2(ctx, a, axis);
  return launch_pass_f4(ctx, a, axis);
}

// One pass along `axis` over `fields` (nullptr: the context's fields).
static int run_pass(atus_ctx *ctx, int axis, int t1, int op, int t2, const NLArgs *nl, int half,
                    void *const *fields = nullptr, int nfields = -1) {
  PassArgs a;
  memset(&a, 0, sizeof(a));
  const int nf = nfields < 0 ? ctx->ncomp : nfields;
  for (int c = 0; c < MAXC; c++) a.psi[c] = (c < nf) ? (fields ? fields[c] : ctx->psi[c]) : nullptr;
  a.t1 = t1;
  a.op = op;
  a.t2 = t2;
  a.per_comp = (op != OP_NL) ? 1 : 0;
  a.nc = (op == OP_NL) ? nf : 1;
  if (op == OP_KIN)
    for (int c = 0; c < MAXC; c++)
      for (int ax = 0; ax < 3; ax++) a.kt[c][ax] = (c < ctx->ncomp) ? ctx->kt[half ? 0 : 1][c][ax] : nullptr;
  a.s_f = scale_fak(ctx->dim, ctx->d);
  a.s_b = scale_fak(ctx->dim, ctx->dk);
  if (nl) a.nl = *nl;
  // per-component passes launch ncomp CTAs in y; override when the field set differs
  if (a.per_comp && nf != ctx->ncomp) {
    int saved = ctx->ncomp;
    ctx->ncomp = nf;
    int r = dispatch_pass(ctx, a, axis, 1);
    ctx->ncomp = saved;
    return r;
  }
  const int tc = a.per_comp ? 1 : tc_for(nf);
  return dispatch_pass(ctx, a, axis, tc);
}

#define RUN(x)                  \
  do {                          \
    int _r = (x);               \
    if (_r != ATUS_OK) return _r; \
  } while (0)

// Forward (dir -1) or inverse (+1) transform of the axes other than 0.
static int transform_inner(atus_ctx *ctx, int dir, void *const *f = nullptr, int nf = -1) {
  if (ctx->dim == 2) return run_pass(ctx, 1, dir, OP_NONE, T_NONE, nullptr, 0, f, nf);
  if (ctx->dim == 3) {
    if (dir == T_FWD) {
      RUN(run_pass(ctx, 2, T_FWD, OP_NONE, T_NONE, nullptr, 0, f, nf));
      return run_pass(ctx, 1, T_FWD, OP_NONE, T_NONE, nullptr, 0, f, nf);
    }
    RUN(run_pass(ctx, 1, T_INV, OP_NONE, T_NONE, nullptr, 0, f, nf));
    return run_pass(ctx, 2, T_INV, OP_NONE, T_NONE, nullptr, 0, f, nf);
  }
  return ATUS_OK;
}

static int grid_blocks(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  return (int)(b < 148 * 16 ? b : 148 * 16);
}

// ------------------------------------------------------------------ long 1D axes (four-step)
// x[n], n = n2c * r + c (r < n1 along view axis 0, stride n2c; c < n2c along
// view axis 1, contiguous).  Forward: transform along r, times W_N^{r' c}
// (r' the transformed index), transform along c; element (k1, k2) then holds
// X[k1 + n1 k2].  Inverse: the same steps backwards with conjugate twiddles.
template <typename R>
__global__ void fs_twiddle_kernel(void *psi, const double2 *tw, int64_t n2c, int64_t N, int conj_) {
  cplx<R> *p = static_cast<cplx<R> *>(psi);
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < N; l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = l / n2c, c = l % n2c;
    double2 w = tw[(r * c) % N];
    if (conj_) w.y = -w.y;
    p[l] = from_d<R>(cmul(to_d<R>(p[l]), w));
  }
}

// Kinetic factor of the four-step spectrum: element (k1, k2) is wavenumber
// index k1 + n1 k2 of the 1D table, with the transform scales applied as in
// the passes: ((u s_f) K) s_b in FP64.
template <typename R>
__global__ void fs_kin_kernel(void *psi, const double2 *kt, int64_t n1, int64_t n2c, double s_f, double s_b) {
  cplx<R> *p = static_cast<cplx<R> *>(psi);
  const int64_t N = n1 * n2c;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < N; l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k1 = l / n2c, k2 = l % n2c;
    const double2 K = kt[k1 + n1 * k2];
    double2 u = to_d<R>(p[l]);
    u.x *= s_f;
    u.y *= s_f;
    u = cmul(u, K);
    u.x *= s_b;
    u.y *= s_b;
    p[l] = from_d<R>(u);
  }
}

// Four-step spectrum <-> natural wavenumber order, FP64 buffers:
// to_natural: dst[k1 + n1 k2] = src[k1 n2c + k2]; else the inverse.
__global__ void fs_reorder_kernel(const double2 *src, double2 *dst, int64_t n1, int64_t n2c, int to_natural) {
  const int64_t N = n1 * n2c;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < N; l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k1 = l / n2c, k2 = l % n2c;
    if (to_natural) dst[k1 + n1 * k2] = src[l];
    else dst[l] = src[k1 + n1 * k2];
  }
}

// The context seen as its n1 x n2c four-step grid while plain transforms run.
struct FsView {
  atus_ctx *c;
  int dim;
  int64_t n[3];
  int lg[3];
  explicit FsView(atus_ctx *ctx) : c(ctx), dim(ctx->dim) {
    for (int a = 0; a < 3; a++) {
      n[a] = ctx->n[a];
      lg[a] = ctx->lg[a];
    }
    ctx->dim = 2;
    ctx->n[0] = ctx->fs_n1;
    ctx->n[1] = ctx->fs_n2;
    ctx->n[2] = 1;
    ctx->lg[0] = ilog2(ctx->fs_n1);
    ctx->lg[1] = ilog2(ctx->fs_n2);
    ctx->lg[2] = 0;
  }
  ~FsView() {
    c->dim = dim;
    for (int a = 0; a < 3; a++) {
      c->n[a] = n[a];
      c->lg[a] = lg[a];
    }
  }
};

static int fs_twiddle(atus_ctx *ctx, void *const *f, int nf, int conj_, bool fp64) {
  for (int i = 0; i < nf; i++) {
    if (fp64)
      fs_twiddle_kernel<double><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(f[i], ctx->fs_tw, ctx->fs_n2,
                                                                                       ctx->npts, conj_);
    else
      fs_twiddle_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(f[i], ctx->fs_tw, ctx->fs_n2,
                                                                                      ctx->npts, conj_);
    LAUNCHED(ctx);
  }
  return ATUS_OK;
}

// Unscaled forward / inverse transform of nf fields (four-step order in k).
static int fs_forward(atus_ctx *ctx, void *const *f, int nf) {
  const bool fp64 = ctx->prec == ATUS_PREC_FP64;
  {
    FsView v(ctx);
    RUN(run_pass(ctx, 0, T_FWD, OP_NONE, T_NONE, nullptr, 0, f, nf));
  }
  RUN(fs_twiddle(ctx, f, nf, 0, fp64));
  FsView v(ctx);
  return run_pass(ctx, 1, T_FWD, OP_NONE, T_NONE, nullptr, 0, f, nf);
}
static int fs_inverse(atus_ctx *ctx, void *const *f, int nf) {
  const bool fp64 = ctx->prec == ATUS_PREC_FP64;
  {
    FsView v(ctx);
    RUN(run_pass(ctx, 1, T_INV, OP_NONE, T_NONE, nullptr, 0, f, nf));
  }
  RUN(fs_twiddle(ctx, f, nf, 1, fp64));
  FsView v(ctx);
  return run_pass(ctx, 0, T_INV, OP_NONE, T_NONE, nullptr, 0, f, nf);
}

// An FP64 four-step spectrum (scratch-sized buffer) into / out of natural order.
static int fs_reorder(atus_ctx *ctx, void *&buf, int to_natural) {
  if (!ctx->fs_tmp) CK(cudaMalloc(&ctx->fs_tmp, 16 * ctx->npts));
  fs_reorder_kernel<<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(
      static_cast<const double2 *>(buf), static_cast<double2 *>(ctx->fs_tmp), ctx->fs_n1, ctx->fs_n2, to_natural);
  LAUNCHED(ctx);
  void *t = buf;
  buf = ctx->fs_tmp;
  ctx->fs_tmp = t;
  return ATUS_OK;
}

// k-space kinetic pass along axis 0: FFT_x, phase, IFFT_x (a long 1D axis:
// four-step transforms around the factor of each wavenumber).
static int kinetic_pass(atus_ctx *ctx, int half) {
  if (ctx->fs_tw) {
    RUN(fs_forward(ctx, ctx->psi, ctx->ncomp));
    const double s_f = scale_fak(ctx->dim, ctx->d), s_b = scale_fak(ctx->dim, ctx->dk);
    for (int c = 0; c < ctx->ncomp; c++) {
      const double2 *kt = ctx->kt[half ? 0 : 1][c][0];
      if (ctx->prec == ATUS_PREC_FP64)
        fs_kin_kernel<double><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(ctx->psi[c], kt, ctx->fs_n1,
                                                                                    ctx->fs_n2, s_f, s_b);
      else
        fs_kin_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(ctx->psi[c], kt, ctx->fs_n1,
                                                                                   ctx->fs_n2, s_f, s_b);
      LAUNCHED(ctx);
    }
    return fs_inverse(ctx, ctx->psi, ctx->ncomp);
  }
  return run_pass(ctx, 0, T_FWD, OP_KIN, T_INV, nullptr, half);
}

// Rabi balls requested with a block: per component comps[c] (c < ncomp) the
// centres k0[(c * n + m) * dim ..] (m < n), radius thr.
struct RabiReq {
  int ncomp, n;
  int comps[2];
  const double *k0;
  double thr;
};

// The kinetic pass with the Rabi sums of the requested components folded in:
// after FFT_x every axis is in k-space and |psi^|^2 does not see the kinetic
// phase, so the sums of the state after the pass are taken there.  Unscaled
// sums go to ctx->red_partial (one row per CTA), the totals to sums[c*n+m].
// ATUS_E_UNSUPPORTED (fields untouched) where the register-staged x pass does
// not apply.
static int kinetic_pass_rabi(atus_ctx *ctx, int half, const RabiReq &rr, double *sums) {
  if (!ctx->use_pass2 || ctx->dim < 2 || ctx->n[0] < 32 || ctx->n[0] > 256) return ATUS_E_UNSUPPORTED;
  PassArgs a;
  memset(&a, 0, sizeof(a));
  for (int c = 0; c < MAXC; c++) a.psi[c] = (c < ctx->ncomp) ? ctx->psi[c] : nullptr;
  a.t1 = T_FWD;
  a.op = OP_KIN;
  a.t2 = T_INV;
  a.per_comp = 1;
  a.nc = 1;
  for (int c = 0; c < MAXC; c++)
    for (int ax = 0; ax < 3; ax++) a.kt[c][ax] = (c < ctx->ncomp) ? ctx->kt[half ? 0 : 1][c][ax] : nullptr;
  a.s_f = scale_fak(ctx->dim, ctx->d);
  a.s_b = scale_fak(ctx->dim, ctx->dk);
  a.rabi_ncomp = rr.ncomp;
  a.rabi_n = rr.n;
  for (int c = 0; c < rr.ncomp; c++) {
    a.rabi_comp[c] = rr.comps[c];
    for (int m = 0; m < rr.n; m++)
      for (int ax = 0; ax < 3; ax++)
        a.rabi_k0[c * rr.n + m][ax] = (ax < ctx->dim) ? rr.k0[(c * rr.n + m) * ctx->dim + ax] : 0.0;
  }
  a.rabi_thr = rr.thr;
  a.rabi_partial = ctx->red_partial;
  CK(cudaMemsetAsync(ctx->red_partial, 0, sizeof(double) * RED_BLOCKS * RED_MAXQ, ctx->stream));
  const int r = (ctx->prec == ATUS_PREC_FP64) ? launch_pass2_d_kr(ctx, a, 0) : launch_pass2_f_kr(ctx, a, 0);
  if (r != ATUS_OK) return r;
  const int nq = rr.ncomp * rr.n;
  reduce_final<<<1, 32, 0, ctx->stream>>>(ctx->red_partial, RED_BLOCKS, nq, ctx->red_out);
  LAUNCHED(ctx);
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red_out, sizeof(double) * nq, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int q = 0; q < nq; q++) sums[q] = ctx->h_red[q];
  return ATUS_OK;
}

// Real-space potential pass: 2D one pass over rows; 3D inverse y, rows, forward y.
static int potential_pass(atus_ctx *ctx, const NLArgs &nl) {
  const int last = ctx->dim - 1;
  if (ctx->dim == 3) RUN(run_pass(ctx, 1, T_INV, OP_NONE, T_NONE, nullptr, 0));
  RUN(run_pass(ctx, last, T_INV, OP_NL, T_FWD, &nl, 0));
  if (ctx->dim == 3) RUN(run_pass(ctx, 1, T_FWD, OP_NONE, T_NONE, nullptr, 0));
  return ATUS_OK;
}

// ------------------------------------------------------------------ reductions
static int reduce(atus_ctx *ctx, RedArgs &a, double *out) {
  a.g = geo(ctx);
  a.dim = ctx->dim;
  for (int ax = 0; ax < 3; ax++) {
    a.d[ax] = ctx->d[ax];
    a.dk[ax] = ctx->dk[ax];
    a.n[ax] = (int)ctx->n[ax];
    a.shift[ax] = (int)(ctx->n[ax] / 2);
  }
  if (ctx->prec == ATUS_PREC_FP64 || a.mode == RED_MOM || a.mode == RED_RABI)
    reduce_kernel<double><<<RED_BLOCKS, RED_THREADS, 0, ctx->stream>>>(a, ctx->red_partial);
  else
    reduce_kernel<float><<<RED_BLOCKS, RED_THREADS, 0, ctx->stream>>>(a, ctx->red_partial);
  LAUNCHED(ctx);
  reduce_final<<<1, 32, 0, ctx->stream>>>(ctx->red_partial, RED_BLOCKS, a.nq, ctx->red_out);
  LAUNCHED(ctx);
  CK(cudaMemcpyAsync(ctx->h_red, ctx->red_out, sizeof(double) * a.nq, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < a.nq; i++) out[i] = ctx->h_red[i];
  return ATUS_OK;
}

// The same reduction, result left in device memory (no host round trip).
static int reduce_dev(atus_ctx *ctx, RedArgs &a, double *dst) {
  a.g = geo(ctx);
  a.dim = ctx->dim;
  for (int ax = 0; ax < 3; ax++) {
    a.d[ax] = ctx->d[ax];
    a.dk[ax] = ctx->dk[ax];
    a.n[ax] = (int)ctx->n[ax];
    a.shift[ax] = (int)(ctx->n[ax] / 2);
  }
  reduce_kernel<double><<<RED_BLOCKS, RED_THREADS, 0, ctx->stream>>>(a, ctx->red_partial);
  LAUNCHED(ctx);
  reduce_final<<<1, 32, 0, ctx->stream>>>(ctx->red_partial, RED_BLOCKS, a.nq, dst);
  LAUNCHED(ctx);
  return ATUS_OK;
}

// Copy component comp into the FP64 scratch buffer (complex128).
static int to_scratch(atus_ctx *ctx, int comp) {
  if (ctx->prec == ATUS_PREC_FP64) {
    CK(cudaMemcpyAsync(ctx->scratch, ctx->psi[comp], 16 * ctx->npts, cudaMemcpyDeviceToDevice, ctx->stream));
  } else {
    convert_out_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>((double2 *)ctx->scratch,
                                                                                     ctx->psi[comp], ctx->npts);
    LAUNCHED(ctx);
  }
  return ATUS_OK;
}

// Forward transform (with the reference's forward scale, applied by the caller)
// of the FP64 scratch buffer over all axes.
static int scratch_forward(atus_ctx *ctx) {
  const int saved = ctx->prec;
  ctx->prec = ATUS_PREC_FP64;
  void *f[1] = {ctx->scratch};
  int r = ATUS_OK;
  if (ctx->fs_tw) {
    r = fs_forward(ctx, f, 1);
    if (r == ATUS_OK) r = fs_reorder(ctx, ctx->scratch, 1);
  } else {
    for (int ax = ctx->dim - 1; ax >= 0 && r == ATUS_OK; ax--)
      r = run_pass(ctx, ax, T_FWD, OP_NONE, T_NONE, nullptr, 0, f, 1);
  }
  ctx->prec = saved;
  return r;
}

// Embedding: a field on a smaller grid with the same spacing, centred in a
// larger one (index offsets (nd - ns) / 2 per axis, both grids centred at
// x = 0), zero outside.
struct EmbedArgs {
  const double2 *src;
  double2 *dst;
  int ns[3], nd[3], off[3];
  int64_t npts_s;
};
__global__ void embed_kernel(EmbedArgs a) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < a.npts_s; l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i2 = l % a.ns[2], i1 = (l / a.ns[2]) % a.ns[1], i0 = l / ((int64_t)a.ns[2] * a.ns[1]);
    const int64_t f = ((i0 + a.off[0]) * a.nd[1] + (i1 + a.off[1])) * a.nd[2] + (i2 + a.off[2]);
    a.dst[f] = a.src[l];
  }
}

// psi *= fak in FP64 (the scale pass of cft_Nd::ft)
template <typename R>
__global__ void ft_scale_kernel(void *psi, double fak, int64_t n) {
  cplx<R> *p = static_cast<cplx<R> *>(psi);
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    const cplx<R> v = p[l];
    p[l] = mk<R>((R)((double)v.x * fak), (R)((double)v.y * fak));
  }
}

// ------------------------------------------------------------------ API
extern "C" {

int atus_create(const atus_grid *grid, int ncomp, int precision, atus_ctx **out) {
  if (!grid || !out) return ATUS_E_ARG;
  *out = nullptr;
  if (grid->dim < 1 || grid->dim > 3 || ncomp < 1 || ncomp > MAXC) return ATUS_E_ARG;
  if (precision != ATUS_PREC_FP64 && precision != ATUS_PREC_MIXED) return ATUS_E_ARG;
  atus_ctx *ctx = new atus_ctx();
  ctx->dim = grid->dim;
  ctx->ncomp = ncomp;
  ctx->prec = precision;
  ctx->csize = precision == ATUS_PREC_FP64 ? 16 : 8;
  ctx->npts = 1;
  for (int a = 0; a < 3; a++) {
    ctx->n[a] = (a < grid->dim) ? grid->n[a] : 1;
    ctx->d[a] = (a < grid->dim) ? grid->d[a] : 0.0;
    ctx->dk[a] = (a < grid->dim) ? grid->dk[a] : 0.0;
    // the longest pass instantiation is 8192 points; a 1D axis up to 2^26
    // points runs as four-step transforms over two such passes
    const int64_t nmax = (grid->dim == 1 && a == 0) ? (int64_t(1) << 26) : 8192;
    if (ctx->n[a] < 1 || (ctx->n[a] & (ctx->n[a] - 1)) != 0 || ctx->n[a] > nmax) {
      delete ctx;
      return ATUS_E_UNSUPPORTED;
    }
    if (a < grid->dim && ctx->n[a] < 2) {
      delete ctx;
      return ATUS_E_UNSUPPORTED;
    }
    ctx->lg[a] = ilog2(ctx->n[a]);
    ctx->npts *= ctx->n[a];
  }
  if (grid->dim == 1) { ctx->ar = ctx->d[0]; ctx->ar_k = ctx->dk[0]; }
  else if (grid->dim == 2) { ctx->ar = ctx->d[0] * ctx->d[1]; ctx->ar_k = ctx->dk[0] * ctx->dk[1]; }
  else { ctx->ar = ctx->d[0] * ctx->d[1] * ctx->d[2]; ctx->ar_k = ctx->dk[0] * ctx->dk[1] * ctx->dk[2]; }
  ctx->t = grid->t;
  {
    // ATUS_PASS2=0: tile kernel only (A/B comparisons of the two pass kernels)
    const char *p2 = getenv("ATUS_PASS2");
    ctx->use_pass2 = !(p2 && p2[0] == '0');
    // ATUS_CLUSTER1D=0: 1D blocks on one CTA only (A/B comparisons)
    const char *c1 = getenv("ATUS_CLUSTER1D");
    ctx->use_cluster1d = !(c1 && c1[0] == '0');
    // ATUS_TMA=0: strided 256-point passes load their tiles themselves (no TMA)
    const char *tm = getenv("ATUS_TMA");
    ctx->use_tma = !(tm && tm[0] == '0');
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { delete ctx; return ATUS_E_CUDA; }
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete ctx; return ATUS_E_CUDA; }
  ctx->stream = ctx->own_stream;
  bool ok = true;
  for (int c = 0; c < ncomp && ok; c++) {
    ok = cudaMalloc(&ctx->psi[c], ctx->csize * ctx->npts) == cudaSuccess;
    if (ok) ok = cudaMemset(ctx->psi[c], 0, ctx->csize * ctx->npts) == cudaSuccess;
  }
  if (ok) ok = cudaMalloc(&ctx->scratch, 16 * ctx->npts) == cudaSuccess;
  if (ok) ok = cudaMalloc(&ctx->err_dev, sizeof(int)) == cudaSuccess && cudaMemset(ctx->err_dev, 0, sizeof(int)) == cudaSuccess;
  if (ok) ok = cudaMalloc(&ctx->red_partial, sizeof(double) * RED_BLOCKS * RED_MAXQ) == cudaSuccess;
  if (ok) ok = cudaMalloc(&ctx->red_out, sizeof(double) * RED_MAXQ) == cudaSuccess;
  if (ok) ok = cudaMallocHost(&ctx->h_red, sizeof(double) * RED_MAXQ) == cudaSuccess;
  if (ok) ok = cudaMallocHost(&ctx->h_sob, sizeof(SobDev)) == cudaSuccess;
  if (ok) {
    ok = cudaMalloc(&ctx->tw64, 16 * TWN) == cudaSuccess;
    if (ok) {
      auto t = twiddles<double>();
      ok = cudaMemcpy(ctx->tw64, t.data(), 16 * TWN, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    ctx->tw = ctx->tw64;
    if (ok && precision == ATUS_PREC_MIXED) {
      // float4 (hi, lo) split of the FP64 table for the compensated FP32 multiply
      ok = cudaMalloc(&ctx->tw, sizeof(float4) * TWN) == cudaSuccess;
      if (ok) {
        const auto t = twiddles<double>();
        std::vector<float4> t4(TWN);
        for (int m = 0; m < TWN; m++) {
          t4[m].x = (float)t[m].x;
          t4[m].y = (float)t[m].y;
          t4[m].z = (float)(t[m].x - (double)t4[m].x);
          t4[m].w = (float)(t[m].y - (double)t4[m].y);
        }
        ok = cudaMemcpy(ctx->tw, t4.data(), sizeof(float4) * TWN, cudaMemcpyHostToDevice) == cudaSuccess;
      }
    }
  }
  if (!ok) {
    atus_destroy(ctx);
    return ATUS_E_NOMEM;
  }
  // CRT_Base's constructor builds the tables once (alpha still zero).
  if (ok && ctx->dim == 1 && ctx->n[0] > 8192) {
    // four-step view n1 x n2 (n2 >= n1, both powers of two <= 8192) and the
    // exact twiddles W_N^m = exp(-2 pi i m / N) rounded once from long double
    const int l = ctx->lg[0];
    ctx->fs_n1 = int64_t(1) << (l / 2);
    ctx->fs_n2 = ctx->n[0] / ctx->fs_n1;
    std::vector<double2> t(ctx->n[0]);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int64_t m = 0; m < ctx->n[0]; m++) {
      const long double th = two_pi * (long double)m / (long double)ctx->n[0];
      t[m].x = (double)cosl(th);
      t[m].y = (double)(-sinl(th));
    }
    ok = cudaMalloc(&ctx->fs_tw, sizeof(double2) * ctx->n[0]) == cudaSuccess &&
         cudaMemcpy(ctx->fs_tw, t.data(), sizeof(double2) * ctx->n[0], cudaMemcpyHostToDevice) == cudaSuccess;
    if (!ok) {
      atus_destroy(ctx);
      return ATUS_E_NOMEM;
    }
  }
  int r = build_kinetic(ctx);
  if (r != ATUS_OK) {
    atus_destroy(ctx);
    return r;
  }
  *out = ctx;
  return ATUS_OK;
}

void atus_destroy(atus_ctx *ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (int c = 0; c < MAXC; c++) {
    cudaFree(ctx->psi[c]);
    cudaFree(ctx->V[c]);
    cudaFree(ctx->sob_lap[c]);
    cudaFree(ctx->sob_psi[c]);
    cudaFree(ctx->sob_grad[c]);
    for (int hf = 0; hf < 2; hf++)
      for (int ax = 0; ax < 3; ax++) cudaFree(ctx->kt[hf][c][ax]);
  }
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
  cudaFree(ctx->snap);
  if (ctx->snap_taken) cudaEventDestroy(ctx->snap_taken);
  if (ctx->snap_read) cudaEventDestroy(ctx->snap_read);
  if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
  cudaFree(ctx->fs_tw);
  cudaFree(ctx->fs_tmp);
  cudaFree(ctx->err_dev);
  cudaFree(ctx->scratch);
  cudaFree(ctx->sob_dev);
  if (ctx->sob_graph) cudaGraphExecDestroy(ctx->sob_graph);
  if (ctx->h_sob) cudaFreeHost(ctx->h_sob);
  if (ctx->tw != ctx->tw64) cudaFree(ctx->tw);
  cudaFree(ctx->tw64);
  cudaFree(ctx->red_partial);
  cudaFree(ctx->red_out);
  if (ctx->h_red) cudaFreeHost(ctx->h_red);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
}

const char *atus_last_error(const atus_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// The device error word after kernels with bounded waits (the TMA-fed
// passes): read once they are done, reset, and reported as ATUS_E_CUDA.
static int wait_check(atus_ctx *ctx) {
  if (!ctx->err_armed) return ATUS_OK;
  ctx->err_armed = false;
  int e = 0;
  CK(cudaMemcpyAsync(&e, ctx->err_dev, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (e == 0) return ATUS_OK;
  CK(cudaMemsetAsync(ctx->err_dev, 0, sizeof(int), ctx->stream));
  return fail(ctx, ATUS_E_CUDA, "a TMA tile copy did not complete within the wait limit");
}

int atus_set_stream(atus_ctx *ctx, void *stream) {
  if (!ctx) return ATUS_E_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return ATUS_OK;
}

int atus_synchronize(atus_ctx *ctx) {
  if (!ctx) return ATUS_E_ARG;
  CK(cudaStreamSynchronize(ctx->stream));
  return wait_check(ctx);
}

int atus_launch_count(const atus_ctx *ctx, int64_t *out) {
  if (!ctx || !out) return ATUS_E_ARG;
  *out = ctx->launches;
  return ATUS_OK;
}

int atus_set_alpha(atus_ctx *ctx, int comp, const double *alpha) {
  if (!ctx || !alpha || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  for (int a = 0; a < 3; a++) ctx->alpha[comp][a] = (a < ctx->dim) ? alpha[a] : 0.0;
  return ATUS_OK;
}

int atus_set_dt(atus_ctx *ctx, double dt) {
  if (!ctx) return ATUS_E_ARG;
  ctx->dt = dt;
  return build_kinetic(ctx);
}

int atus_get_dt(const atus_ctx *ctx, double *dt) {
  if (!ctx || !dt) return ATUS_E_ARG;
  *dt = ctx->dt;
  return ATUS_OK;
}

int atus_set_wait_limits(atus_ctx *ctx, int64_t wait_rounds, int drop_copies) {
  if (!ctx || wait_rounds < 1 || (drop_copies != 0 && drop_copies != 1)) return ATUS_E_ARG;
  ctx->wait_limit = (long)wait_rounds;
  ctx->drop_copies = drop_copies;
  return ATUS_OK;
}

int atus_set_bragg_stable(atus_ctx *ctx, int on) {
  if (!ctx || (on != 0 && on != 1)) return ATUS_E_ARG;
  ctx->bragg_stable = on;
  return ATUS_OK;
}

int atus_set_time(atus_ctx *ctx, double t) {
  if (!ctx) return ATUS_E_ARG;
  ctx->t = t;
  return ATUS_OK;
}

int atus_get_time(const atus_ctx *ctx, double *t) {
  if (!ctx || !t) return ATUS_E_ARG;
  *t = ctx->t;
  return ATUS_OK;
}

int atus_set_gs(atus_ctx *ctx, const double *gs) {
  if (!ctx || !gs) return ATUS_E_ARG;
  for (int i = 0; i < MAXC * MAXC; i++) ctx->gs[i] = 0;
  for (int i = 0; i < ctx->ncomp; i++)
    for (int j = 0; j < ctx->ncomp; j++) ctx->gs[i * MAXC + j] = gs[j + ctx->ncomp * i];
  return ATUS_OK;
}

int atus_clone(const atus_ctx *src, atus_ctx **out) {
  if (!src || !out) return ATUS_E_ARG;
  *out = nullptr;
  atus_grid g{};
  g.dim = src->dim;
  for (int ax = 0; ax < 3; ax++) {
    g.n[ax] = src->n[ax];
    g.d[ax] = src->d[ax];
    g.dk[ax] = src->dk[ax];
  }
  g.t = src->t;
  atus_ctx *ctx = nullptr;
  const int r = atus_create(&g, src->ncomp, src->prec, &ctx);
  if (r != ATUS_OK) return r;
  // the source's work must be complete before its buffers are read
  if (cudaStreamSynchronize(src->stream) != cudaSuccess) {
    atus_destroy(ctx);
    return ATUS_E_CUDA;
  }
  ctx->t = src->t;
  ctx->dt = src->dt;
  memcpy(ctx->alpha, src->alpha, sizeof(ctx->alpha));
  memcpy(ctx->gs, src->gs, sizeof(ctx->gs));
  ctx->laser = src->laser;
  ctx->laser2 = src->laser2;
  ctx->win_t0 = src->win_t0;
  ctx->win_dur[0] = src->win_dur[0];
  ctx->win_dur[1] = src->win_dur[1];
  ctx->bragg_stable = src->bragg_stable;
  ctx->use_pass2 = src->use_pass2;
  ctx->use_cluster1d = src->use_cluster1d;
  ctx->use_tma = src->use_tma;
  int e = ATUS_OK;
  auto copy = [&](void *dst, const void *from, size_t bytes) {
    if (e == ATUS_OK && cudaMemcpyAsync(dst, from, bytes, cudaMemcpyDeviceToDevice, ctx->stream) != cudaSuccess)
      e = fail(ctx, ATUS_E_CUDA, "clone copy");
  };
  for (int c = 0; c < src->ncomp; c++) {
    copy(ctx->psi[c], src->psi[c], src->csize * src->npts);
    if (src->V[c]) {
      if (cudaMalloc(&ctx->V[c], sizeof(double) * src->npts) != cudaSuccess) e = ATUS_E_NOMEM;
      else copy(ctx->V[c], src->V[c], sizeof(double) * src->npts);
    }
    // the kinetic phases as the source holds them (built for its dt and the
    // alpha it had then)
    for (int hf = 0; hf < 2; hf++)
      for (int ax = 0; ax < 3; ax++)
        if (src->kt[hf][c][ax]) copy(ctx->kt[hf][c][ax], src->kt[hf][c][ax], sizeof(double2) * src->n[ax]);
  }
  if (e == ATUS_OK && cudaStreamSynchronize(ctx->stream) != cudaSuccess) e = ATUS_E_CUDA;
  if (e != ATUS_OK) {
    atus_destroy(ctx);
    return e;
  }
  *out = ctx;
  return ATUS_OK;
}

int atus_set_potential(atus_ctx *ctx, int comp, const double *V) {
  if (!ctx || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  if (!V) {
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(ctx->V[comp]);
    ctx->V[comp] = nullptr;
    return ATUS_OK;
  }
  if (!ctx->V[comp] && cudaMalloc(&ctx->V[comp], sizeof(double) * ctx->npts) != cudaSuccess)
    return fail(ctx, ATUS_E_NOMEM, "potential allocation");
  CK(cudaMemcpyAsync(ctx->V[comp], V, sizeof(double) * ctx->npts, cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return ATUS_OK;
}

int atus_set_laser(atus_ctx *ctx, const atus_laser *laser) {
  if (!ctx || !laser) return ATUS_E_ARG;
  ctx->laser = *laser;
  return ATUS_OK;
}

int atus_set_laser2(atus_ctx *ctx, const atus_laser *laser2) {
  if (!ctx || !laser2) return ATUS_E_ARG;
  ctx->laser2 = *laser2;
  return ATUS_OK;
}

int atus_set_pulse_windows(atus_ctx *ctx, double t_start, const double *duration) {
  if (!ctx || !duration) return ATUS_E_ARG;
  ctx->win_t0 = t_start;
  ctx->win_dur[0] = duration[0];
  ctx->win_dur[1] = duration[1];
  return ATUS_OK;
}

int atus_upload_psi(atus_ctx *ctx, int comp, const double *psi) {
  if (!ctx || !psi || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  if (ctx->prec == ATUS_PREC_FP64) {
    CK(cudaMemcpyAsync(ctx->psi[comp], psi, 16 * ctx->npts, cudaMemcpyHostToDevice, ctx->stream));
  } else {
    CK(cudaMemcpyAsync(ctx->scratch, psi, 16 * ctx->npts, cudaMemcpyHostToDevice, ctx->stream));
    convert_in_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(ctx->psi[comp],
                                                                                    (const double2 *)ctx->scratch, ctx->npts);
    LAUNCHED(ctx);
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return ATUS_OK;
}

int atus_download_psi(atus_ctx *ctx, int comp, double *psi) {
  if (!ctx || !psi || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  if (ctx->prec == ATUS_PREC_FP64) {
    CK(cudaMemcpyAsync(psi, ctx->psi[comp], 16 * ctx->npts, cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    RUN(to_scratch(ctx, comp));
    CK(cudaMemcpyAsync(psi, ctx->scratch, 16 * ctx->npts, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CK(cudaStreamSynchronize(ctx->stream));
  return ATUS_OK;
}

// ------------------------------------------------------------------ asynchronous output
// The copy into the staging buffer runs on the context's stream (ordered after
// the steps before it) and returns at once; the device->host copies run on a
// copy stream of the context, from whichever host thread asks for them, so the
// steps enqueued next overlap them.
int atus_snapshot(atus_ctx *ctx) {
  if (!ctx) return ATUS_E_ARG;
  if (!ctx->snap) {
    CK(cudaMalloc(&ctx->snap, (size_t)16 * ctx->npts * ctx->ncomp));
    CK(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ctx->snap_taken, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ctx->snap_read, cudaEventDisableTiming));
  }
  // the staging buffer may still be read by the copies of the last snapshot
  CK(cudaStreamWaitEvent(ctx->stream, ctx->snap_read, 0));
  for (int c = 0; c < ctx->ncomp; c++) {
    double2 *dst = static_cast<double2 *>(ctx->snap) + (size_t)c * ctx->npts;
    if (ctx->prec == ATUS_PREC_FP64) {
      CK(cudaMemcpyAsync(dst, ctx->psi[c], 16 * ctx->npts, cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
      convert_out_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(dst, ctx->psi[c], ctx->npts);
      LAUNCHED(ctx);
    }
  }
  CK(cudaEventRecord(ctx->snap_taken, ctx->stream));
  return ATUS_OK;
}

int atus_snapshot_read(atus_ctx *ctx, int comp, double *host_dst) {
  if (!ctx || !host_dst || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  if (!ctx->snap) return fail(ctx, ATUS_E_ARG, "no snapshot taken");
  cudaStream_t s = ctx->copy_stream;
  // wait on the host until the staging copy is done: a copy into pageable
  // memory queued behind it would hold up the context's other launches
  cudaError_t e = cudaEventSynchronize(ctx->snap_taken);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(host_dst, static_cast<double2 *>(ctx->snap) + (size_t)comp * ctx->npts, 16 * ctx->npts,
                        cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaEventRecord(ctx->snap_read, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? ATUS_OK : ATUS_E_CUDA;
}

int atus_device_psi(atus_ctx *ctx, int comp, void **dptr) {
  if (!ctx || !dptr || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  *dptr = ctx->psi[comp];
  return ATUS_OK;
}

// cft_Nd::ft (cft_1d.cpp:61-77, cft_2d.cpp:58-74, cft_3d.cpp:58-74) on one
// component: the unnormalised transform over every axis (isign -1: FFTW's
// forward sign, +1: backward), then the scale pass with (dx/sqrt(2 pi))^dim
// after a forward and (dk/sqrt(2 pi))^dim after a backward transform.
int atus_ft(atus_ctx *ctx, int comp, int isign) {
  if (!ctx || comp < 0 || comp >= ctx->ncomp || (isign != -1 && isign != 1)) return ATUS_E_ARG;
  void *f[1] = {ctx->psi[comp]};
  const int dir = (isign < 0) ? T_FWD : T_INV;
  if (ctx->fs_tw) {
    // the spectrum in natural wavenumber order, as cft_1d::ft leaves it
    if (ctx->prec != ATUS_PREC_FP64) return fail(ctx, ATUS_E_UNSUPPORTED, "ft of a long complex64 1D field");
    if (isign < 0) {
      RUN(fs_forward(ctx, f, 1));
      RUN(fs_reorder(ctx, ctx->psi[comp], 1));
    } else {
      RUN(fs_reorder(ctx, ctx->psi[comp], 0));
      void *g[1] = {ctx->psi[comp]};
      RUN(fs_inverse(ctx, g, 1));
    }
  } else {
    for (int ax = ctx->dim - 1; ax >= 0; ax--) RUN(run_pass(ctx, ax, dir, OP_NONE, T_NONE, nullptr, 0, f, 1));
  }
  const double fak = scale_fak(ctx->dim, isign < 0 ? ctx->d : ctx->dk);
  if (ctx->prec == ATUS_PREC_FP64)
    ft_scale_kernel<double><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(ctx->psi[comp], fak, ctx->npts);
  else
    ft_scale_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(ctx->psi[comp], fak, ctx->npts);
  LAUNCHED(ctx);
  return wait_check(ctx);
}

int atus_embed(atus_ctx *src, int comp_s, atus_ctx *dst, int comp_d) {
  if (!src || !dst || comp_s < 0 || comp_s >= src->ncomp || comp_d < 0 || comp_d >= dst->ncomp) return ATUS_E_ARG;
  atus_ctx *ctx = dst;
  if (src->prec != ATUS_PREC_FP64 || dst->prec != ATUS_PREC_FP64)
    return fail(dst, ATUS_E_UNSUPPORTED, "embedding needs FP64 contexts");
  if (src->dim != dst->dim) return fail(dst, ATUS_E_ARG, "grids of different dimension");
  EmbedArgs a;
  for (int ax = 0; ax < 3; ax++) {
    if (dst->n[ax] < src->n[ax]) return fail(dst, ATUS_E_ARG, "the target grid has fewer points");
    if (ax < src->dim && fabs(src->d[ax] - dst->d[ax]) > 1e-12 * dst->d[ax])
      return fail(dst, ATUS_E_ARG, "grids of different spacing");
    a.ns[ax] = (int)src->n[ax];
    a.nd[ax] = (int)dst->n[ax];
    a.off[ax] = (int)((dst->n[ax] - src->n[ax]) / 2);
  }
  {  // the source field must be complete before the target stream reads it
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, src->stream));
    CK(cudaStreamWaitEvent(dst->stream, ev, 0));
    cudaEventDestroy(ev);
  }
  CK(cudaMemsetAsync(dst->psi[comp_d], 0, 16 * dst->npts, dst->stream));
  a.src = static_cast<const double2 *>(src->psi[comp_s]);
  a.dst = static_cast<double2 *>(dst->psi[comp_d]);
  a.npts_s = src->npts;
  embed_kernel<<<grid_blocks(src->npts, 256), 256, 0, dst->stream>>>(a);
  LAUNCHED(dst);
  CK(cudaStreamSynchronize(dst->stream));
  return ATUS_OK;
}

int atus_ft_step(atus_ctx *ctx, int half) {
  if (!ctx) return ATUS_E_ARG;
  RUN(transform_inner(ctx, T_FWD));
  RUN(kinetic_pass(ctx, half));
  RUN(transform_inner(ctx, T_INV));
  ctx->t += half ? 0.5 * ctx->dt : ctx->dt;
  return wait_check(ctx);
}

static int check_kind(atus_ctx *ctx, int kind) {
  if (kind < K_NL || kind > K_RAMAN) return fail(ctx, ATUS_E_ARG, "unknown step kind");
  if (kind == K_NL_IF2 && (ctx->ncomp % 2) != 0)
    return fail(ctx, ATUS_E_ARG, "the two-species freeprop needs an even number of components");
  if (kind == K_BRAGG_DS && ctx->ncomp != 4) return fail(ctx, ATUS_E_ARG, "the two-species bragg_ad needs four components");
  if (kind == K_NUM_BRAGG && (ctx->ncomp < 2 || ctx->ncomp > 3))
    return fail(ctx, ATUS_E_ARG, "the numerical bragg step needs two or three components");
  if (kind == K_RAMAN && ctx->ncomp != 3) return fail(ctx, ATUS_E_ARG, "the raman step needs three components");
  if (kind == K_BRAGG && ctx->ncomp != 2) return fail(ctx, ATUS_E_ARG, "bragg_ad needs two components");
  if (kind == K_DBRAGG && ctx->ncomp != 3) return fail(ctx, ATUS_E_ARG, "the three-level bragg_ad needs three components");
  return ATUS_OK;
}

int atus_nl_step(atus_ctx *ctx, int kind, double F) {
  if (!ctx) return ATUS_E_ARG;
  RUN(check_kind(ctx, kind));
  NLKArgs a;
  memset(&a, 0, sizeof(a));
  for (int c = 0; c < MAXC; c++) a.psi[c] = ctx->psi[c];
  a.nl = nl_args(ctx, kind, ctx->t + 0.5 * ctx->dt, F);
  a.g = geo(ctx);
  if (ctx->prec == ATUS_PREC_FP64)
    nl_kernel<double><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(a);
  else
    nl_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(a);
  LAUNCHED(ctx);
  return ATUS_OK;
}

static int strang_block(atus_ctx *ctx, int nk, int kind, const double *F, const RabiReq *rr, double *sums,
                        bool *fused);

int atus_strang_block(atus_ctx *ctx, int nk, int kind, const double *F) {
  RUN(strang_block(ctx, nk, kind, F, nullptr, nullptr, nullptr));
  return wait_check(ctx);
}

int atus_strang_block_rabi(atus_ctx *ctx, int nk, int kind, const double *F, int ncomp_r, const int *comps,
                           const double *k0, int n, double thr, double *out) {
  if (!ctx || !out || !comps || !k0 || ncomp_r < 1 || ncomp_r > 2 || n < 1 || ncomp_r * n > RED_MAXQ)
    return ATUS_E_ARG;
  for (int c = 0; c < ncomp_r; c++)
    if (comps[c] < 0 || comps[c] >= ctx->ncomp) return ATUS_E_ARG;
  RabiReq rr;
  rr.ncomp = ncomp_r;
  rr.n = n;
  rr.comps[0] = comps[0];
  rr.comps[1] = ncomp_r > 1 ? comps[1] : -1;
  rr.k0 = k0;
  rr.thr = thr;
  double sums[RED_MAXQ];
  bool fused = false;
  RUN(strang_block(ctx, nk, kind, F, &rr, sums, &fused));
  RUN(wait_check(ctx));
  if (!fused) {  // the separate transform and reduction of compute_rabi_integrals
    for (int c = 0; c < ncomp_r; c++)
      RUN(atus_rabi_integrals_comp(ctx, comps[c], k0 + (size_t)c * n * ctx->dim, n, thr, out + c * n));
    return ATUS_OK;
  }
  const double f = scale_fak(ctx->dim, ctx->d);
  for (int q = 0; q < ncomp_r * n; q++) out[q] = ctx->ar_k * (f * f * sums[q]);
  return ATUS_OK;
}

static int strang_block(atus_ctx *ctx, int nk, int kind, const double *F, const RabiReq *rr, double *sums,
                        bool *fused) {
  if (!ctx || nk < 1) return ATUS_E_ARG;
  RUN(check_kind(ctx, kind));
  const double dt = ctx->dt;
  // shared memory of the resident 1D kernel (padded pencils, Pad<N>)
  const int64_t n0 = ctx->n[0];
  const int64_t np1d = ((n0 >= 16) ? (n0 + n0 / 16) : n0) | 1;
  const bool on_cluster = ctx->use_cluster1d && n0 >= 2048 && n0 <= 8192;  // cluster1d.cuh
  const bool fits1d = on_cluster || (int64_t)ctx->csize * tc_for(ctx->ncomp) * np1d <= 227 * 1024;
  if (ctx->dim == 1 && ctx->ncomp <= 2 && kind != K_NUM_BRAGG && !ctx->fs_tw && fits1d) {
    Block1DArgs a;
    memset(&a, 0, sizeof(a));
    for (int c = 0; c < MAXC; c++) {
      a.psi[c] = ctx->psi[c];
      a.kh[c] = (c < ctx->ncomp) ? ctx->kt[0][c][0] : nullptr;
      a.kf[c] = (c < ctx->ncomp) ? ctx->kt[1][c][0] : nullptr;
    }
    a.s_f = scale_fak(ctx->dim, ctx->d);
    a.s_b = scale_fak(ctx->dim, ctx->dk);
    a.tw = ctx->tw;
    a.nl = nl_args(ctx, kind, 0.0, 1.0);
    a.nk = nk;
    a.t0 = ctx->t;
    double *dF = nullptr;
    if (F) {
      CK(cudaMalloc(&dF, sizeof(double) * nk));
      CK(cudaMemcpyAsync(dF, F, sizeof(double) * nk, cudaMemcpyHostToDevice, ctx->stream));
    }
    a.F = dF;
    const int tc = tc_for(ctx->ncomp);
    int r;
    if (tc > 2) return fail(ctx, ATUS_E_UNSUPPORTED, "1D blocks take at most two components");
    if (ctx->prec == ATUS_PREC_FP64)
      r = tc == 1 ? launch_block1d_d1(ctx, a) : launch_block1d_d2(ctx, a);
    else
      r = tc == 1 ? launch_block1d_f1(ctx, a) : launch_block1d_f2(ctx, a);
    if (dF) {
      cudaStreamSynchronize(ctx->stream);
      cudaFree(dF);
    }
    if (r == ATUS_OK) {
      // replay the header-time additions of the reference
      double t = ctx->t + 0.5 * dt;
      for (int j = 0; j < nk; j++) t += (j == nk - 1) ? 0.5 * dt : dt;
      ctx->t = t;
      return ATUS_OK;
    }
    // ATUS_E_UNSUPPORTED: nothing was launched (no cluster placeable, the
    // field too long for one CTA); the per-step passes below run the block
    if (r != ATUS_E_UNSUPPORTED) return r;
    ctx->err.clear();
  }
  if (ctx->dim == 1) {
    // more components or points than the resident 1D kernel holds, or a step
    // that reads the header time itself: per step one kinetic pass (FFT,
    // phase, IFFT per component) and one point-wise potential step
    RUN(kinetic_pass(ctx, 1));
    ctx->t += 0.5 * dt;
    for (int j = 0; j < nk; j++) {
      NLKArgs a;
      memset(&a, 0, sizeof(a));
      for (int c = 0; c < MAXC; c++) a.psi[c] = ctx->psi[c];
      a.nl = nl_args(ctx, kind, ctx->t + 0.5 * dt, F ? F[j] : 1.0);
      a.g = geo(ctx);
      if (ctx->prec == ATUS_PREC_FP64)
        nl_kernel<double><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(a);
      else
        nl_kernel<float><<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>(a);
      LAUNCHED(ctx);
      const bool last = (j == nk - 1);
      RUN(kinetic_pass(ctx, last ? 1 : 0));
      ctx->t += last ? 0.5 * dt : dt;
    }
    return ATUS_OK;
  }
  // 2D / 3D: [inner forward] kinetic(half) { potential, kinetic } ... [inner inverse]
  RUN(transform_inner(ctx, T_FWD));
  RUN(kinetic_pass(ctx, 1));
  ctx->t += 0.5 * dt;
  for (int j = 0; j < nk; j++) {
    const NLArgs nl = nl_args(ctx, kind, ctx->t + 0.5 * dt, F ? F[j] : 1.0);
    RUN(potential_pass(ctx, nl));
    const bool last = (j == nk - 1);
    int r = ATUS_E_UNSUPPORTED;
    if (last && rr) {
      r = kinetic_pass_rabi(ctx, 1, *rr, sums);
      if (r == ATUS_OK && fused) *fused = true;
    }
    if (r == ATUS_E_UNSUPPORTED) r = kinetic_pass(ctx, last ? 1 : 0);
    RUN(r);
    ctx->t += last ? 0.5 * dt : dt;
  }
  return transform_inner(ctx, T_INV);
}

int atus_profile_passes(atus_ctx *ctx, int kind, int reps, double *ms, double *lps, double *bytes, int *npass) {
  if (!ctx || !ms || !lps || !bytes || !npass || reps < 1) return ATUS_E_ARG;
  RUN(check_kind(ctx, kind));
  // The passes run out of the Strang schedule (a kinetic pass alone carries
  // the whole transform scale, so repeated launches can drive complex64
  // fields to zero): the fields and the time are saved here and put back.
  const size_t fbytes = (size_t)ctx->csize * (size_t)ctx->npts;
  char *saved = nullptr;
  CK(cudaMalloc(&saved, fbytes * ctx->ncomp));
  cudaError_t ce = cudaSuccess;
  for (int c = 0; c < ctx->ncomp && ce == cudaSuccess; c++)
    ce = cudaMemcpyAsync(saved + c * fbytes, ctx->psi[c], fbytes, cudaMemcpyDeviceToDevice, ctx->stream);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaStreamSynchronize(ctx->stream);
    cudaFree(saved);
    return cuda_check(ctx, ce, "profile_passes: saving the fields");
  }
  const double t_saved = ctx->t;
  const NLArgs nl = nl_args(ctx, kind, ctx->t + 0.5 * ctx->dt, 1.0);
  const double fb = 2.0 * (double)ctx->csize * (double)ctx->ncomp * (double)ctx->npts;  // read + write all fields
  const double vb = (kind == K_NL) ? 8.0 * ctx->npts * [&] {
    int k = 0;
    for (int c = 0; c < ctx->ncomp; c++) k += ctx->V[c] != nullptr;
    return k;
  }() : 0.0;
  int np = 0;
  auto timed = [&](auto &&launch, double per_step, double b) -> int {
    RUN(launch());  // warm-up launch
    CK(cudaEventRecord(e0, ctx->stream));
    for (int r = 0; r < reps; r++) RUN(launch());
    CK(cudaEventRecord(e1, ctx->stream));
    CK(cudaEventSynchronize(e1));
    float t = 0;
    CK(cudaEventElapsedTime(&t, e0, e1));
    ms[np] = (double)t / reps;
    lps[np] = per_step;
    bytes[np] = b;
    np++;
    return ATUS_OK;
  };
  int r = ATUS_OK;
  if (ctx->dim == 1) {
    const int nk = 16;
    auto blk = [&]() { return atus_strang_block(ctx, nk, kind, nullptr); };
    r = timed(blk, 1.0 / nk, fb);
  } else {
    auto kin = [&]() { return kinetic_pass(ctx, 0); };
    r = timed(kin, 1.0, fb);
    const int last = ctx->dim - 1;
    if (r == ATUS_OK && ctx->dim == 3) {
      auto yinv = [&]() { return run_pass(ctx, 1, T_INV, OP_NONE, T_NONE, nullptr, 0); };
      r = timed(yinv, 1.0, fb);
    }
    if (r == ATUS_OK) {
      auto pot = [&]() { return run_pass(ctx, last, T_INV, OP_NL, T_FWD, &nl, 0); };
      r = timed(pot, 1.0, fb + vb);
    }
    if (r == ATUS_OK && ctx->dim == 3) {
      auto yfwd = [&]() { return run_pass(ctx, 1, T_FWD, OP_NONE, T_NONE, nullptr, 0); };
      r = timed(yfwd, 1.0, fb);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  for (int c = 0; c < ctx->ncomp && ce == cudaSuccess; c++)
    ce = cudaMemcpyAsync(ctx->psi[c], saved + c * fbytes, fbytes, cudaMemcpyDeviceToDevice, ctx->stream);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
  cudaFree(saved);
  ctx->t = t_saved;
  *npass = np;
  if (ce != cudaSuccess) return cuda_check(ctx, ce, "profile_passes: restoring the fields");
  return r;
}

int atus_particle_number(atus_ctx *ctx, int comp, double *out) {
  if (!ctx || !out || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  RedArgs a;
  memset(&a, 0, sizeof(a));
  a.mode = RED_NORM;
  a.nq = 1;
  a.a = ctx->psi[comp];
  double s;
  RUN(reduce(ctx, a, &s));
  *out = ctx->ar * s;
  return ATUS_OK;
}

int atus_expval_position(atus_ctx *ctx, int comp, double *out) {
  if (!ctx || !out || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  RedArgs a;
  memset(&a, 0, sizeof(a));
  a.mode = RED_POS;
  a.nq = ctx->dim;
  a.a = ctx->psi[comp];
  double s[3];
  RUN(reduce(ctx, a, s));
  for (int i = 0; i < ctx->dim; i++) out[i] = ctx->ar * s[i];
  return ATUS_OK;
}

int atus_expval_momentum(atus_ctx *ctx, int comp, double *out) {
  if (!ctx || !out || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  RUN(to_scratch(ctx, comp));
  RUN(scratch_forward(ctx));
  RedArgs a;
  memset(&a, 0, sizeof(a));
  a.mode = RED_MOM;
  a.nq = ctx->dim;
  a.a = ctx->scratch;
  double s[3];
  RUN(reduce(ctx, a, s));
  const double f = scale_fak(ctx->dim, ctx->d);
  for (int i = 0; i < ctx->dim; i++) out[i] = ctx->ar_k * (f * f * s[i]);
  return wait_check(ctx);
}

int atus_setup_momentum(atus_ctx *ctx, int comp, const double *p) {
  if (!ctx || !p || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  double pp[3] = {0, 0, 0};
  for (int i = 0; i < ctx->dim; i++) pp[i] = p[i];
  const Geo g = geo(ctx);
  const int b = grid_blocks(ctx->npts, 256);
  if (ctx->prec == ATUS_PREC_FP64)
    momentum_kernel<double><<<b, 256, 0, ctx->stream>>>(ctx->psi[comp], g, pp[0], pp[1], pp[2], ctx->d[0], ctx->d[1],
                                                         ctx->d[2], (int)(ctx->n[0] / 2), (int)(ctx->n[1] / 2),
                                                         (int)(ctx->n[2] / 2));
  else
    momentum_kernel<float><<<b, 256, 0, ctx->stream>>>(ctx->psi[comp], g, pp[0], pp[1], pp[2], ctx->d[0], ctx->d[1],
                                                        ctx->d[2], (int)(ctx->n[0] / 2), (int)(ctx->n[1] / 2),
                                                        (int)(ctx->n[2] / 2));
  LAUNCHED(ctx);
  return ATUS_OK;
}

int atus_rabi_integrals(atus_ctx *ctx, const double *k0, int n, double thr, double *out) {
  return atus_rabi_integrals_comp(ctx, 0, k0, n, thr, out);
}

int atus_rabi_integrals_comp(atus_ctx *ctx, int comp, const double *k0, int n, double thr, double *out) {
  if (!ctx || !out || n < 0 || n > RED_MAXQ || (n > 0 && !k0)) return ATUS_E_ARG;
  if (comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  if (n == 0) return ATUS_OK;
  RUN(to_scratch(ctx, comp));
  RUN(scratch_forward(ctx));
  RedArgs a;
  memset(&a, 0, sizeof(a));
  a.mode = RED_RABI;
  a.nq = n;
  a.a = ctx->scratch;
  a.thr = thr;
  for (int m = 0; m < n; m++)
    for (int ax = 0; ax < 3; ax++) a.k0[m][ax] = (ax < ctx->dim) ? k0[m * ctx->dim + ax] : 0.0;
  double s[RED_MAXQ];
  RUN(reduce(ctx, a, s));
  const double f = scale_fak(ctx->dim, ctx->d);
  for (int m = 0; m < n; m++) out[m] = ctx->ar_k * (f * f * s[m]);
  return wait_check(ctx);
}

// ------------------------------------------------------------------ Sobolev gradient
// Real k-space filter of an FP64 buffer over all axes: forward transforms,
// filter inside the axis-0 pass, inverse transforms.
static int sob_filter_n(atus_ctx *ctx, void *const *bufs, int nb, int mode, double alpha) {
  if (ctx->fs_tw) return fail(ctx, ATUS_E_UNSUPPORTED, "the Sobolev filter takes 1D grids of at most 8192 points");
  const int saved = ctx->prec;
  ctx->prec = ATUS_PREC_FP64;
  int r = ATUS_OK;
  for (int ax = ctx->dim - 1; ax >= 1 && r == ATUS_OK; ax--) r = run_pass(ctx, ax, T_FWD, OP_NONE, T_NONE, nullptr, 0, bufs, nb);
  if (r == ATUS_OK) {
    PassArgs a;
    memset(&a, 0, sizeof(a));
    for (int k = 0; k < nb; k++) a.psi[k] = bufs[k];
    a.t1 = T_FWD;
    a.op = OP_FILT;
    a.t2 = T_INV;
    a.per_comp = 1;
    a.nc = 1;
    a.filt_mode = mode;
    a.filt_alpha = alpha;
    a.filt_scale = round_trip_scale(ctx);
    const int saved_nc = ctx->ncomp;
    ctx->ncomp = nb;
    r = dispatch_pass(ctx, a, 0, 1);
    ctx->ncomp = saved_nc;
  }
  for (int ax = 1; ax < ctx->dim && r == ATUS_OK; ax++) r = run_pass(ctx, ax, T_INV, OP_NONE, T_NONE, nullptr, 0, bufs, nb);
  ctx->prec = saved;
  return r;
}

static int sob_filter(atus_ctx *ctx, void *buf, int mode, double alpha) {
  void *f[1] = {buf};
  return sob_filter_n(ctx, f, 1, mode, alpha);
}

static int sob_norms(atus_ctx *ctx, double *N) {
  for (int i = 0; i < ctx->ncomp; i++) RUN(atus_particle_number(ctx, i, &N[i]));
  return ATUS_OK;
}

static int sob_renorm(atus_ctx *ctx) {
  double N[MAXC];
  RUN(sob_norms(ctx, N));
  for (int i = 0; i < ctx->ncomp; i++) {
    scale_kernel<<<grid_blocks(ctx->npts, 256), 256, 0, ctx->stream>>>((double2 *)ctx->psi[i], 1.0 / sqrt(N[i]), ctx->npts);
    LAUNCHED(ctx);
  }
  return ATUS_OK;
}

static int sob_laplace(atus_ctx *ctx) {
  for (int i = 0; i < ctx->ncomp; i++) {
    CK(cudaMemcpyAsync(ctx->sob_lap[i], ctx->psi[i], 16 * ctx->npts, cudaMemcpyDeviceToDevice, ctx->stream));
    RUN(sob_filter(ctx, ctx->sob_lap[i], FILT_LAPLACE, ctx->sob_alpha[i]));
  }
  return ATUS_OK;
}

static int sob_iterate_once(atus_ctx *ctx, double *res_out, double *N_out) {
  const int n = ctx->ncomp;
  const int blocks = grid_blocks(ctx->npts, 256);
  for (int i = 0; i < n; i++) {  // Compute_Sobolev_Psi
    CK(cudaMemcpyAsync(ctx->sob_psi[i], ctx->psi[i], 16 * ctx->npts, cudaMemcpyDeviceToDevice, ctx->stream));
    RUN(sob_filter(ctx, ctx->sob_psi[i], FILT_SOBOLEV, ctx->sob_alpha[i]));
  }
  RUN(sob_laplace(ctx));  // Compute_Laplace
  for (int i = 0; i < n; i++) {  // Compute_Sobolev_Gradient
    SobArgs a;
    memset(&a, 0, sizeof(a));
    for (int j = 0; j < MAXC; j++) a.psi[j] = (const double2 *)ctx->psi[j];
    a.lap = (const double2 *)ctx->sob_lap[i];
    a.V = ctx->V[i];
    a.grad = (double2 *)ctx->sob_grad[i];
    a.comp = i;
    a.ncomp = n;
    for (int k = 0; k < MAXC * MAXC; k++) a.gs[k] = ctx->gs[k];
    a.npts = ctx->npts;
    sob_assemble_kernel<<<blocks, 256, 0, ctx->stream>>>(a);
    LAUNCHED(ctx);
    RUN(sob_filter(ctx, ctx->sob_grad[i], FILT_SOBOLEV, ctx->sob_alpha[i]));
  }
  for (int i = 0; i < n; i++) {  // Project_Sobolev_Gradient
    RedArgs r;
    memset(&r, 0, sizeof(r));
    r.mode = RED_DOT2;
    r.nq = 2;
    r.a = ctx->psi[i];
    r.b = ctx->sob_grad[i];
    r.c = ctx->sob_psi[i];
    double q[2];
    RUN(reduce(ctx, r, q));
    const double fak = q[0] / q[1];
    axpy_kernel<<<blocks, 256, 0, ctx->stream>>>((double2 *)ctx->sob_grad[i], (const double2 *)ctx->sob_psi[i], fak,
                                                 ctx->npts);
    LAUNCHED(ctx);
  }
  double res_tot = 0;  // Compute_res
  for (int i = 0; i < n; i++) {
    RedArgs r;
    memset(&r, 0, sizeof(r));
    r.mode = RED_NORM;
    r.nq = 1;
    r.a = ctx->sob_grad[i];
    double q;
    RUN(reduce(ctx, r, &q));
    q *= ctx->ar;
    res_tot += q * q;
  }
  res_tot = sqrt(res_tot);
  double N[MAXC];
  RUN(sob_norms(ctx, N));
  bool renorm = false;
  for (int i = 0; i < n; i++) {
    if (N_out) N_out[i] = N[i];
    if (fabs(N[i] - 1) > 1e-5) renorm = true;
  }
  if (renorm) RUN(sob_renorm(ctx));
  for (int i = 0; i < n; i++) {
    axpy_kernel<<<blocks, 256, 0, ctx->stream>>>((double2 *)ctx->psi[i], (const double2 *)ctx->sob_grad[i],
                                                 ctx->stepsize, ctx->npts);
    LAUNCHED(ctx);
  }
  if (res_out) *res_out = res_tot;
  return ATUS_OK;
}

// One iteration of sob_iterate_once with every scalar in device memory:
// the same kernels and reductions in the same order; psi changes only in an
// active iteration (not yet converged, below max_iter).
static int sob_iterate_dev(atus_ctx *ctx) {
  // The reference's gradient S(-Lap psi + W psi), W = V + sum_j g_ij |psi_j|^2,
  // S = 1/(1 + alpha k^2), taken as S(W psi) + psi - S psi: S alpha k^2 = 1 - S,
  // so the Laplacian's transforms drop out (two filters per component instead
  // of three; the same quantities up to rounding).
  const int n = ctx->ncomp;
  const int blocks = grid_blocks(ctx->npts, 256);
  SobDev *d = (SobDev *)ctx->sob_dev;
  for (int i = 0; i < n; i++) {  // S psi (Compute_Sobolev_Psi) and S(W psi), filtered together
    SobArgs a;  // W psi into the gradient buffer, psi into the Sobolev buffer, one pass
    memset(&a, 0, sizeof(a));
    for (int j = 0; j < MAXC; j++) a.psi[j] = (const double2 *)ctx->psi[j];
    a.lap = nullptr;
    a.V = ctx->V[i];
    a.grad = (double2 *)ctx->sob_grad[i];
    a.copy = (double2 *)ctx->sob_psi[i];
    a.comp = i;
    a.ncomp = n;
    for (int k = 0; k < MAXC * MAXC; k++) a.gs[k] = ctx->gs[k];
    a.npts = ctx->npts;
    sob_assemble_kernel<<<blocks, 256, 0, ctx->stream>>>(a);
    LAUNCHED(ctx);
    void *bufs[2] = {ctx->sob_psi[i], ctx->sob_grad[i]};
    RUN(sob_filter_n(ctx, bufs, 2, FILT_SOBOLEV, ctx->sob_alpha[i]));
  }
  for (int i = 0; i < n; i++) {
    RedArgs r;  // G = S(W psi) + psi - S psi, the projection's two products and <psi, psi> in one pass
    memset(&r, 0, sizeof(r));
    r.mode = RED_SOBG;
    r.nq = 3;
    r.a = ctx->psi[i];
    r.c = ctx->sob_psi[i];
    r.w = (double2 *)ctx->sob_grad[i];
    RUN(reduce_dev(ctx, r, d->q[i]));
    RedArgs p;  // Project_Sobolev_Gradient fused with the norm of the projected gradient
    memset(&p, 0, sizeof(p));
    p.mode = RED_PROJ;
    p.nq = 1;
    p.w = (double2 *)ctx->sob_grad[i];
    p.c = ctx->sob_psi[i];
    p.fq = d->q[i];
    RUN(reduce_dev(ctx, p, &d->g2[i]));
  }
  sob_scalars_kernel<<<1, 1, 0, ctx->stream>>>(d, ctx->ar, n);
  LAUNCHED(ctx);
  for (int i = 0; i < n; i++) {
    sob_update_kernel<<<blocks, 256, 0, ctx->stream>>>((double2 *)ctx->psi[i], (const double2 *)ctx->sob_grad[i],
                                                      ctx->stepsize, d, i, ctx->npts);
    LAUNCHED(ctx);
  }
  sob_commit_kernel<<<1, 1, 0, ctx->stream>>>(d);
  LAUNCHED(ctx);
  return ATUS_OK;
}

int atus_sob_init(atus_ctx *ctx, const double *alpha, double stepsize) {
  if (!ctx || !alpha) return ATUS_E_ARG;
  if (ctx->prec != ATUS_PREC_FP64) return fail(ctx, ATUS_E_UNSUPPORTED, "the Sobolev descent runs in FP64");
  for (int i = 0; i < ctx->ncomp; i++) {
    ctx->sob_alpha[i] = alpha[i];
    if (!ctx->sob_lap[i]) {
      if (cudaMalloc(&ctx->sob_lap[i], 16 * ctx->npts) != cudaSuccess ||
          cudaMalloc(&ctx->sob_psi[i], 16 * ctx->npts) != cudaSuccess ||
          cudaMalloc(&ctx->sob_grad[i], 16 * ctx->npts) != cudaSuccess)
        return fail(ctx, ATUS_E_NOMEM, "Sobolev buffers");
    }
  }
  ctx->stepsize = stepsize;
  ctx->sob_ready = true;
  return ATUS_OK;
}

int atus_sob_renormalize(atus_ctx *ctx) {
  if (!ctx || !ctx->sob_ready) return ctx ? fail(ctx, ATUS_E_STATE, "atus_sob_init first") : ATUS_E_ARG;
  return sob_renorm(ctx);
}

int atus_sob_iterate(atus_ctx *ctx, int n_iter, double *res, double *N) {
  if (!ctx || !ctx->sob_ready) return ctx ? fail(ctx, ATUS_E_STATE, "atus_sob_init first") : ATUS_E_ARG;
  for (int k = 0; k < n_iter; k++) RUN(sob_iterate_once(ctx, res, N));
  return wait_check(ctx);
}

// Iterations until the residual is <= epsilon (the reference's run loop, the
// update of the converging iteration included) or max_iter.  The first
// iteration runs directly, the rest as a CUDA graph of SOB_CHUNK device-side
// iterations; the host reads the device scalars once per chunk.
constexpr int SOB_CHUNK = 64;

int atus_sob_run(atus_ctx *ctx, double epsilon, int max_iter, int *iters, double *res) {
  if (!ctx || !ctx->sob_ready) return ctx ? fail(ctx, ATUS_E_STATE, "atus_sob_init first") : ATUS_E_ARG;
  if (max_iter < 1) return fail(ctx, ATUS_E_ARG, "max_iter < 1");
  RUN(sob_renorm(ctx));
  if (!ctx->sob_dev) CK(cudaMalloc(&ctx->sob_dev, sizeof(SobDev)));
  SobDev h;
  memset(&h, 0, sizeof(h));
  h.eps = epsilon;
  h.max_iter = max_iter;
  CK(cudaMemcpyAsync(ctx->sob_dev, &h, sizeof(SobDev), cudaMemcpyHostToDevice, ctx->stream));
  RUN(sob_iterate_dev(ctx));  // eager: kernel attributes are set outside any capture
  if (ctx->sob_graph && ctx->sob_graph_step != ctx->stepsize) {
    cudaGraphExecDestroy(ctx->sob_graph);
    ctx->sob_graph = nullptr;
  }
  if (!ctx->sob_graph) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    int r = ATUS_OK;
    for (int k = 0; k < SOB_CHUNK && r == ATUS_OK; k++) r = sob_iterate_dev(ctx);
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (r != ATUS_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      return r != ATUS_OK ? r : cuda_check(ctx, e, "Sobolev graph capture");
    }
    const cudaError_t ie = cudaGraphInstantiate(&ctx->sob_graph, g, 0);
    cudaGraphDestroy(g);
    CK(ie);
    ctx->sob_graph_step = ctx->stepsize;
  }
  SobDev *hd = reinterpret_cast<SobDev *>(ctx->h_sob);
  for (;;) {
    CK(cudaMemcpyAsync(hd, ctx->sob_dev, sizeof(SobDev), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (hd->done || hd->iters >= max_iter) break;
    CK(cudaGraphLaunch(ctx->sob_graph, ctx->stream));
  }
  if (iters) *iters = hd->iters;
  if (res) *res = hd->res;
  return wait_check(ctx);
}

int atus_sob_mu(atus_ctx *ctx, double *mu) {
  if (!ctx || !mu || !ctx->sob_ready) return ctx ? fail(ctx, ATUS_E_STATE, "atus_sob_init first") : ATUS_E_ARG;
  RUN(sob_laplace(ctx));
  for (int i = 0; i < ctx->ncomp; i++) {
    RedArgs r;
    memset(&r, 0, sizeof(r));
    r.mode = RED_MU;
    r.nq = 1;
    r.a = ctx->psi[i];
    r.b = ctx->sob_lap[i];
    r.V = ctx->V[i];
    for (int j = 0; j < MAXC; j++) r.psi_all[j] = ctx->psi[j];
    r.ncomp = ctx->ncomp;
    r.comp = i;
    for (int k = 0; k < MAXC * MAXC; k++) r.gs[k] = ctx->gs[k];
    double q;
    RUN(reduce(ctx, r, &q));
    mu[i] = ctx->ar * q;
  }
  return ATUS_OK;
}

}  // extern "C"

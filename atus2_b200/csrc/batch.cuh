// batch.cuh -- kernels of the batched sweep: many independent two-component
// Bragg instances (parameter sweeps over pulse area, detuning, interaction
// strength and pulse length) with uneven grids.
//
// 1D instances: batch1d_kernel, one CTA per instance, persistent over the
//   instances of one grid length and over the whole Strang block
//   half, (V, full)^(nk-1), V, half  (include/CRT_Base_IF.h:779-789 with the
//   Bragg step of source/interferometry/src/bragg.cpp:185-304).  RES = 2 keeps
//   both components in shared memory; RES = 1 keeps one and parks the other
//   in global memory (L2), swapping them around each kinetic step -- for
//   grids whose two components do not fit (16384 complex64 points).  The
//   Gaussian pulse envelope F(t) is evaluated on the device.
// 2D instances: batch_pass2_kernel / batch_tile_kernel run one pass (the
//   same passes as a single 2D context) over the tiles of every instance of a
//   size class; the tile of work item w belongs to instance w / tiles.
#pragma once
#include "pass2.cuh"
#include "pass512.cuh"

namespace atus {

// Gaussian pulse envelope exp(-(t - tc)^2 / (2 sigma^2)); two_sigma2 <= 0: 1.
struct Pulse {
  double tc, two_sigma2;
};
__device__ __forceinline__ double pulse_at(const Pulse &p, double t) {
  if (p.two_sigma2 <= 0.0) return 1.0;
  const double u = t - p.tc;
  return exp(-(u * u) / p.two_sigma2);
}

// Bragg coupling of complex64 instances: FP64 phase arguments reduced modulo
// 2 pi, FP32 cos / sincos -- coupling accurate to FP32 for FP32 fields.  FP64
// instances use bragg_coupling (kernels.cuh).
__device__ __forceinline__ void bragg_coupling_mixed(const NLArgs &a, double x0, double &Omega, double &ec,
                                                     double &es) {
  const double t1 = a.t1;
  const double arg =
      a.L.laser_k0 * x0 - (a.L.laser_domh0 + a.L.chirp * t1 + a.L.chirp_rate0 * t1) * t1 + a.L.phase0 / 2;
  Omega = a.F * a.L.Amp0 * (double)cosf((float)reduce_2pi(arg));
  float s, c;
  sincosf((float)reduce_2pi(-0.5 * (a.L.laser_dk0 * x0)), &s, &c);
  ec = c;
  es = s;
}

template <typename R>
__device__ __forceinline__ void coupling_at(const NLArgs &a, double x0, double &om, double &ec, double &es) {
  if constexpr (sizeof(R) == 8) bragg_coupling(a, x0, om, ec, es);
  else bragg_coupling_mixed(a, x0, om, ec, es);
}

// ------------------------------------------------------------------ 1D
struct BInst1 {
  void *psi[2];            // device fields of the instance
  const double2 *kh, *kf;  // half / full kinetic factors (FP64, N entries)
  double s_f, s_b;         // transform scales
  Pulse pulse;
  NLArgs nl;               // Bragg step parameters (kind K_BRAGG, ncomp 2)
};

// psi^ <- ((psi^ s_f) K) s_b, K in FP64 (as kin_1d).
template <typename R, int N, int NT>
__device__ __forceinline__ void b1_kin(cplx<R> *s, const double2 *tab, double s_f, double s_b) {
  for (int i = threadIdx.x; i < N; i += NT) {
    const int si = Pad<N>::idx(0, i);
    double2 v = to_d<R>(s[si]);
    v.x *= s_f;
    v.y *= s_f;
    v = cmul(v, __ldg(&tab[i]));
    v.x *= s_b;
    v.y *= s_b;
    s[si] = from_d<R>(v);
  }
  __syncthreads();
}

// One kinetic step of the component held in s.
template <typename R, int N, int NT>
__device__ __forceinline__ void b1_kinetic(cplx<R> *s, const typename TwTab<R>::type *tw, const double2 *tab,
                                           double s_f, double s_b) {
  fft_tile<R, N, 1, NT, -1, TWN>(s, tw);
  b1_kin<R, N, NT>(s, tab, s_f, s_b);
  fft_tile<R, N, 1, NT, +1, TWN>(s, tw);
}

template <typename R, int N, int NT, int RES>
__device__ __forceinline__ void b1_load(cplx<R> *s, const cplx<R> *src) {
  for (int i = threadIdx.x; i < N; i += NT) s[Pad<N>::idx(0, i)] = src[i];
}
template <typename R, int N, int NT, int RES>
__device__ __forceinline__ void b1_store(const cplx<R> *s, cplx<R> *dst) {
  for (int i = threadIdx.x; i < N; i += NT) dst[i] = s[Pad<N>::idx(0, i)];
}

template <typename R, int N, int NT, int RES>
__global__ void __launch_bounds__(NT) batch1d_kernel(const BInst1 *__restrict__ insts, const int *__restrict__ order,
                                                     const double *__restrict__ t0, int ninst, int nk, const void *twv) {
  // insts and t0 are indexed by batch index; order lists the class's instances
  using C = cplx<R>;
  constexpr int NP = Pad<N>::NP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *const s = reinterpret_cast<C *>(smem_raw);
  const typename TwTab<R>::type *tw = (const typename TwTab<R>::type *)twv;
  // the instance's Bragg parameters live in shared memory (thread 0 sets the
  // step's time and pulse amplitude): a per-thread copy of the ~0.5 KB block
  // sat in local memory
  __shared__ NLArgs s_nl;
  const NLArgs &nl = s_nl;
  for (int k = blockIdx.x; k < ninst; k += gridDim.x) {
    const int id = order[k];
    const BInst1 &in = insts[id];
    C *fld[2] = {(C *)in.psi[0], (C *)in.psi[1]};
    {
      static_assert(sizeof(NLArgs) % 8 == 0, "NLArgs is copied in 8-byte words");
      const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&in.nl);
      unsigned long long *dst = reinterpret_cast<unsigned long long *>(&s_nl);
      for (int e = threadIdx.x; e < (int)(sizeof(NLArgs) / 8); e += NT) dst[e] = src[e];
    }
    __syncthreads();
    const double dt = nl.dt;
    double t = t0[id];
    if constexpr (RES == 2) {
      b1_load<R, N, NT, RES>(s, fld[0]);
      b1_load<R, N, NT, RES>(s + NP, fld[1]);
      __syncthreads();
      b1_kinetic<R, N, NT>(s, tw, in.kh, in.s_f, in.s_b);
      b1_kinetic<R, N, NT>(s + NP, tw, in.kh, in.s_f, in.s_b);
      t += 0.5 * dt;
      for (int j = 0; j < nk; j++) {
        if (threadIdx.x == 0) {
          s_nl.t1 = t + 0.5 * dt;
          s_nl.F = pulse_at(in.pulse, s_nl.t1);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < N; i += NT) {
          const double x0 = (double)(i - nl.shift0) * nl.dx0;
          double om, ec, es;
          coupling_at<R>(nl, x0, om, ec, es);
          C v[MAXC];
          v[0] = s[Pad<N>::idx(0, i)];
          v[1] = s[NP + Pad<N>::idx(0, i)];
          nl_point<R, 2>(nl, v, i, x0, om, ec, es);
          s[Pad<N>::idx(0, i)] = v[0];
          s[NP + Pad<N>::idx(0, i)] = v[1];
        }
        __syncthreads();
        const bool last = (j == nk - 1);
        const double2 *tab = last ? in.kh : in.kf;
        b1_kinetic<R, N, NT>(s, tw, tab, in.s_f, in.s_b);
        b1_kinetic<R, N, NT>(s + NP, tw, tab, in.s_f, in.s_b);
        t += last ? 0.5 * dt : dt;
      }
      b1_store<R, N, NT, RES>(s, fld[0]);
      b1_store<R, N, NT, RES>(s + NP, fld[1]);
    } else {
      // one component resident (index rc), the other in global memory
      int rc = 0;
      b1_load<R, N, NT, RES>(s, fld[0]);
      __syncthreads();
      b1_kinetic<R, N, NT>(s, tw, in.kh, in.s_f, in.s_b);
      b1_store<R, N, NT, RES>(s, fld[0]);
      __syncthreads();
      b1_load<R, N, NT, RES>(s, fld[1]);
      rc = 1;
      __syncthreads();
      b1_kinetic<R, N, NT>(s, tw, in.kh, in.s_f, in.s_b);
      t += 0.5 * dt;
      for (int j = 0; j < nk; j++) {
        if (threadIdx.x == 0) {
          s_nl.t1 = t + 0.5 * dt;
          s_nl.F = pulse_at(in.pulse, s_nl.t1);
        }
        __syncthreads();
        C *other = fld[rc ^ 1];
        for (int i = threadIdx.x; i < N; i += NT) {
          const double x0 = (double)(i - nl.shift0) * nl.dx0;
          double om, ec, es;
          coupling_at<R>(nl, x0, om, ec, es);
          const C res = s[Pad<N>::idx(0, i)], oth = other[i];
          C v[MAXC];
          v[0] = rc ? oth : res;
          v[1] = rc ? res : oth;
          nl_point<R, 2>(nl, v, i, x0, om, ec, es);
          s[Pad<N>::idx(0, i)] = rc ? v[1] : v[0];
          other[i] = rc ? v[0] : v[1];
        }
        __syncthreads();
        const bool last = (j == nk - 1);
        const double2 *tab = last ? in.kh : in.kf;
        b1_kinetic<R, N, NT>(s, tw, tab, in.s_f, in.s_b);
        b1_store<R, N, NT, RES>(s, fld[rc]);
        __syncthreads();
        rc ^= 1;
        b1_load<R, N, NT, RES>(s, fld[rc]);
        __syncthreads();
        b1_kinetic<R, N, NT>(s, tw, tab, in.s_f, in.s_b);
        t += last ? 0.5 * dt : dt;
      }
      b1_store<R, N, NT, RES>(s, fld[rc]);
    }
    __syncthreads();  // shared memory is reused by the next instance
  }
}

// ------------------------------------------------------------------ 2D
// One batched pass: per instance a complete PassArgs (this pass kind, the
// instance's fields, tables and tile counts), the pulse and the header time
// at the start of the block; the potential step `step` of the block uses
// t1 = t0 + dt (step + 1) and F = pulse(t1).
struct BPass {
  const PassArgs *args;  // per instance of the class
  const int *ids;        // batch index of each instance of the class
  const Pulse *pulse;    // per batch index
  const double *t0;      // per batch index
  int ninst;
  int64_t items;   // work items per instance
  int step;
  int potential;   // 1: fill nl.t1 / nl.F for the step
};

// Copies the instance's pass arguments into shared memory (with the step's
// time and pulse amplitude) -- the per-item argument block of the kernels below.
__device__ __forceinline__ void bpass_args(const BPass &bp, int inst, PassArgs *sa) {
  const unsigned long long *src = reinterpret_cast<const unsigned long long *>(bp.args + inst);
  unsigned long long *dst = reinterpret_cast<unsigned long long *>(sa);
  constexpr int W = (int)(sizeof(PassArgs) / 8);
  static_assert(sizeof(PassArgs) % 8 == 0, "PassArgs is copied in 8-byte words");
  for (int e = threadIdx.x; e < W; e += blockDim.x) dst[e] = src[e];
  __syncthreads();
  if (threadIdx.x == 0 && bp.potential) {
    const int id = bp.ids[inst];
    sa->nl.t1 = bp.t0[id] + sa->nl.dt * (double)(bp.step + 1);
    sa->nl.F = pulse_at(bp.pulse[id], sa->nl.t1);
  }
  __syncthreads();
}

template <typename R, int N, int TC, int MODE, bool STRIDED>
__global__ void __launch_bounds__(Tile2<R>::NT, Tile2<R>::MINB) batch_pass2_kernel(BPass bp) {
  using Cfg = P2Cfg<R, N, TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_om[Cfg::B], s_ec[Cfg::B], s_es[Cfg::B];
  __shared__ __align__(16) PassArgs sa;
  bool setup = false;
  const int64_t W = bp.items * bp.ninst;
  for (int64_t w = blockIdx.x; w < W; w += gridDim.x) {
    const int inst = (int)(w / bp.items);
    bpass_args(bp, inst, &sa);
    if (!setup) {  // twiddle rows (the same for every instance of the class)
      p2_setup<R, N, TC, M2_INV>(sa, smem_raw);
      setup = true;
      __syncthreads();  // twiddle rows visible to every warp before the first exchange
    }
    p2_item<R, N, TC, MODE, STRIDED>(sa, tile_geo<Cfg::B, N>(sa, w % bp.items), smem_raw, false, s_om, s_ec,
                                            s_es);
    __syncthreads();  // sa is rewritten by the next item
  }
}

// 512-point register-staged variant (complex64 fields).
template <typename R, int TC, int MODE, bool STRIDED>
__global__ void __launch_bounds__(P5Cfg<R, TC>::NT, 4) batch_pass512_kernel(BPass bp) {
  using Cfg = P5Cfg<R, TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_om[Cfg::B], s_ec[Cfg::B], s_es[Cfg::B];
  __shared__ __align__(16) PassArgs sa;
  bool setup = false;
  const int64_t W = bp.items * bp.ninst;
  for (int64_t w = blockIdx.x; w < W; w += gridDim.x) {
    const int inst = (int)(w / bp.items);
    bpass_args(bp, inst, &sa);
    if (!setup) {
      p5_setup<R, TC>(sa, smem_raw);
      setup = true;
    }
    p5_item<R, TC, MODE, STRIDED>(sa, tile_geo<Cfg::B, 512>(sa, w % bp.items), smem_raw, s_om, s_ec, s_es);
    __syncthreads();
  }
}

// Tile variant (any pencil length): the whole tile is loaded into shared
// memory and transformed with fft_tile (radix-16 Stockham passes), then the
// operator and the second transform, as pass_kernel without the prefetch.
template <typename R, int N, int TC>
struct BTileCfg {
  static constexpr int NT = Tile<R>::NT;
  static constexpr int B0 = Tile<R>::E / (N * TC);
  static constexpr int B = B0 > 0 ? B0 : 1;
  static constexpr int NP = Pad<N>::NP;
  static constexpr size_t smem = sizeof(cplx<R>) * TC * B * NP;
};

template <typename R, int N, int TC, int MODE>
__global__ void __launch_bounds__(Tile<R>::NT) batch_tile_kernel(BPass bp) {
  using C = cplx<R>;
  using Cfg = BTileCfg<R, N, TC>;
  constexpr int B = Cfg::B, NT = Cfg::NT, NP = Cfg::NP;
  static_assert((B * N) % NT == 0, "tile must be a multiple of the CTA size");
  constexpr int LPT = B * N / NT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *const s = reinterpret_cast<C *>(smem_raw);
  __shared__ double s_om[B], s_ec[B], s_es[B];
  __shared__ __align__(16) PassArgs sa;
  const int64_t W = bp.items * bp.ninst;
  for (int64_t w = blockIdx.x; w < W; w += gridDim.x) {
    const int inst = (int)(w / bp.items);
    bpass_args(bp, inst, &sa);
    const PassArgs &a = sa;
    const typename TwTab<R>::type *tw = (const typename TwTab<R>::type *)a.tw;
    const TileGeo g = tile_geo<B, N>(a, w % bp.items);
    const int nc = a.per_comp ? 1 : a.nc;
    #pragma unroll
    for (int c = 0; c < TC; c++) {
      const C *src = (const C *)pick(a.psi, g.comp0 + c);
      #pragma unroll 4
      for (int k = 0; k < LPT; k++) {
        const int r = threadIdx.x + k * NT;
        int b, i;
        if (a.sa > 1) { b = r % B; i = r / B; } else { i = r % N; b = r / N; }
        s[c * B * NP + Pad<N>::idx(b, i)] =
            (c < nc && b < g.nb) ? src[g.base0 + b * g.pstride + (int64_t)i * a.sa] : mk<R>(0, 0);
      }
    }
    __syncthreads();
    if constexpr (MODE == M2_FWD) {
      fft_tile<R, N, TC * B, NT, -1, TWN>(s, tw);
    } else if constexpr (MODE == M2_INV) {
      fft_tile<R, N, TC * B, NT, +1, TWN>(s, tw);
    } else if constexpr (MODE == M2_KIN) {
      fft_tile<R, N, TC * B, NT, -1, TWN>(s, tw);
      const double2 *kx = a.kt[0][0], *ky = a.kt[0][1], *kz = a.kt[0][2];
      #pragma unroll
      for (int c = 1; c < MAXC; c++)
        if (g.comp0 == c) { kx = a.kt[c][0]; ky = a.kt[c][1]; kz = a.kt[c][2]; }
      for (int e = threadIdx.x; e < B * N; e += NT) {
        const int b = e / N, i = e % N;
        if (b < g.nb) {
          const int64_t l = g.base0 + b * g.pstride + (int64_t)i * a.sa;
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
      fft_tile<R, N, TC * B, NT, +1, TWN>(s, tw);
    } else {  // M2_NL
      fft_tile<R, N, TC * B, NT, +1, TWN>(s, tw);
      const bool bragg = (a.nl.kind == K_BRAGG);
      if (bragg && !a.x_along) {
        for (int b = threadIdx.x; b < B; b += NT) {
          double om = 0, ec = 1, es = 0;
          if (b < g.nb) {
            int ix, iy, iz;
            idx3(a.g, g.base0 + b * g.pstride, ix, iy, iz);
            coupling_at<R>(a.nl, (double)(ix - a.nl.shift0) * a.nl.dx0, om, ec, es);
          }
          s_om[b] = om; s_ec[b] = ec; s_es[b] = es;
        }
        __syncthreads();
      }
      for (int e = threadIdx.x; e < B * N; e += NT) {
        const int b = e / N, i = e % N;
        if (b < g.nb) {
          const int64_t l = g.base0 + b * g.pstride + (int64_t)i * a.sa;
          int ix, iy, iz;
          idx3(a.g, l, ix, iy, iz);
          const double x0 = (double)(ix - a.nl.shift0) * a.nl.dx0;
          double om = 0, ec = 1, es = 0;
          if (bragg) {
            if (a.x_along) coupling_at<R>(a.nl, x0, om, ec, es);
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
      fft_tile<R, N, TC * B, NT, -1, TWN>(s, tw);
    }
    #pragma unroll
    for (int c = 0; c < TC; c++) {
      if (c < nc) {
        C *dst = (C *)pick(a.psi, g.comp0 + c);
        #pragma unroll 4
        for (int k = 0; k < LPT; k++) {
          const int r = threadIdx.x + k * NT;
          int b, i;
          if (a.sa > 1) { b = r % B; i = r / B; } else { i = r % N; b = r / N; }
          if (b < g.nb) dst[g.base0 + b * g.pstride + (int64_t)i * a.sa] = s[c * B * NP + Pad<N>::idx(b, i)];
        }
      }
    }
    __syncthreads();
  }
}


// ------------------------------------------------------------------ kernel tables
// Function pointer, threads, dynamic shared memory and (2D) pencils per tile
// of one kernel instantiation, for the host's generic launches.
struct BKernel {
  const void *fn;
  int nt;
  size_t smem;
  int B;
};
// 2D variants: register-staged passes (32..256 points), shared-memory tile
// passes, register-staged 512-point passes (complex64)
enum { BV_P2 = 0, BV_TILE = 1, BV_P5 = 2 };

}  // namespace atus

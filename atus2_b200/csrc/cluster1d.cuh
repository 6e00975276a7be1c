// cluster1d.cuh -- a whole 1D Strang block on a cluster of C = 16 CTAs (16
// SMs) that exchange through distributed shared memory.
//
// N = P x C.  With n = p + P r (r < C) and k = k1 + C k2 (k1 < C):
//
//   X[k1 + C k2] = sum_p W_P^{p k2} W_N^{p k1} sum_r x[p + P r] W_C^{r k1}.
//
// Home layout H: CTA q holds the columns p = q P/C + pl (pl < P/C) for every
// r, so the C-point DFTs over r are local, and so is the potential step
// (point-wise; the x coordinate comes from the global index).  Bin layout K:
// CTA k1 holds y[p][k1] for every p -- one P-point pencil, transformed
// locally (fft_tile) to X[k1 + C k2] at k2, where the kinetic factor of
// wavenumber index k1 + C k2 applies.  A kinetic step is: column DFTs and
// twiddles W_N^{p k1} (local), cluster barrier, H -> K exchange (remote
// reads), P-point FFT, kinetic factor, P-point IFFT, cluster barrier,
// K -> H exchange (remote reads), conjugate twiddles and column IDFTs.  Each
// exchange moves (C - 1)/C of a CTA's values across the cluster; H and K are
// separate buffers, so two barriers per step order every remote read
// against the writes around it (a buffer is rewritten only after the next
// barrier, by which time its readers have moved on).  The last barrier
// before exit keeps every CTA's shared memory alive until the others have
// read it.
#pragma once
#include <cooperative_groups.h>

#include "kernels.cuh"

namespace atus {

// CTAs of the cluster: 16, a non-portable size (the launcher opts in).
// Measured on the 1D 4096-point rt_solver block: 8 CTAs 8.85 us per step,
// 16 CTAs 7.11 us, one CTA 15.9 us.
#define ATUS_C1_CLUSTER 16

template <typename R, int N, int TC>
struct C1Cfg {
  static constexpr int C = ATUS_C1_CLUSTER;
  static constexpr int P = N / C;      // points of a bin pencil
  static constexpr int PC = P / C;     // columns of a CTA
  static constexpr int NT = 256;
  static constexpr int NP = Pad<P>::NP;
  static constexpr int HN = TC * C * PC;  // H values (= TC x P)
  static constexpr size_t smem = sizeof(cplx<R>) * (HN + TC * NP);
};

// One kinetic step (FFT, factor tab of the wavenumber, IFFT) of the TC
// components; H in home layout on entry and exit.
template <typename R, int N, int TC>
__device__ __forceinline__ void c1_kinetic(cooperative_groups::cluster_group &cl, cplx<R> *H, cplx<R> *K,
                                           const typename TwTab<R>::type *tw, const double2 *const (&tab)[TC],
                                           int nc, double s_f, double s_b) {
  using C_ = cplx<R>;
  using Cfg = C1Cfg<R, N, TC>;
  constexpr int C = Cfg::C, P = Cfg::P, PC = Cfg::PC, NT = Cfg::NT, NP = Cfg::NP;
  const int q = (int)cl.block_rank();
  // column DFTs over r and twiddles W_N^{p k1}: H[c][k1][pl] = y[p][k1]
  for (int e = threadIdx.x; e < TC * PC; e += NT) {
    const int c = e / PC, pl = e % PC, p = q * PC + pl;
    C_ v[C];
    #pragma unroll
    for (int r = 0; r < C; r++) v[r] = H[(c * C + r) * PC + pl];
    dftR<C, -1>(v);
    #pragma unroll
    for (int k1 = 1; k1 < C; k1++) v[k1] = twmul<-1>(v[k1], tw[(p * k1) * (TWN / N)]);
    #pragma unroll
    for (int k1 = 0; k1 < C; k1++) H[(c * C + k1) * PC + pl] = v[k1];
  }
  cl.sync();
  // H -> K: bin q of every column, from the CTA that owns the column
  for (int e = threadIdx.x; e < TC * P; e += NT) {
    const int c = e / P, p = e % P;
    const C_ *src = cl.map_shared_rank(H, p / PC);
    K[c * NP + Pad<P>::idx(0, p)] = src[(c * C + q) * PC + p % PC];
  }
  __syncthreads();
  fft_tile<R, P, TC, NT, -1, TWN>(K, tw);
  // psi^ <- ((psi^ s_f) K) s_b in FP64 at wavenumber index q + C k2 (the
  // component loop unrolled: a run-time index into tab would put the
  // pointer array in local memory)
  #pragma unroll
  for (int c = 0; c < TC; c++) {
    if (c < nc) {
      for (int k2 = threadIdx.x; k2 < P; k2 += NT) {
        const int si = c * NP + Pad<P>::idx(0, k2);
        double2 v = to_d<R>(K[si]);
        v.x *= s_f;
        v.y *= s_f;
        v = cmul(v, __ldg(&tab[c][q + C * k2]));
        v.x *= s_b;
        v.y *= s_b;
        K[si] = from_d<R>(v);
      }
    }
  }
  __syncthreads();
  fft_tile<R, P, TC, NT, +1, TWN>(K, tw);
  cl.sync();
  // K -> H: column pl of every bin, from the CTA that owns the bin
  for (int e = threadIdx.x; e < TC * C * PC; e += NT) {
    const int c = e / (C * PC), k1 = (e / PC) % C, pl = e % PC;
    const C_ *src = cl.map_shared_rank(K, k1);
    H[(c * C + k1) * PC + pl] = src[c * NP + Pad<P>::idx(0, q * PC + pl)];
  }
  __syncthreads();
  // conjugate twiddles and column IDFTs: H[c][r][pl] = x[p + P r]
  for (int e = threadIdx.x; e < TC * PC; e += NT) {
    const int c = e / PC, pl = e % PC, p = q * PC + pl;
    C_ v[C];
    v[0] = H[(c * C) * PC + pl];
    #pragma unroll
    for (int k1 = 1; k1 < C; k1++) v[k1] = twmul<+1>(H[(c * C + k1) * PC + pl], tw[(p * k1) * (TWN / N)]);
    dftR<C, +1>(v);
    #pragma unroll
    for (int r = 0; r < C; r++) H[(c * C + r) * PC + pl] = v[r];
  }
  __syncthreads();
}

template <typename R, int N, int TC>
__global__ void __cluster_dims__(ATUS_C1_CLUSTER, 1, 1) __launch_bounds__(256, 1) cluster1d_kernel(Block1DArgs a) {
  using C_ = cplx<R>;
  using Cfg = C1Cfg<R, N, TC>;
  constexpr int C = Cfg::C, P = Cfg::P, PC = Cfg::PC, NT = Cfg::NT;
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  const int q = (int)cl.block_rank();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C_ *const H = reinterpret_cast<C_ *>(smem_raw);
  C_ *const K = H + Cfg::HN;
  const int nc = a.nl.ncomp;
  const typename TwTab<R>::type *tw = (const typename TwTab<R>::type *)a.tw;
  C_ *fld[TC];
  const double2 *kh[TC], *kf[TC];
  #pragma unroll
  for (int c = 0; c < TC; c++) {
    fld[c] = (C_ *)a.psi[c];
    kh[c] = a.kh[c];
    kf[c] = a.kf[c];
  }
  // the CTA's columns: points q PC + pl + P r
  #pragma unroll
  for (int c = 0; c < TC; c++)
    for (int e = threadIdx.x; e < C * PC; e += NT) {
      const int r = e / PC, pl = e % PC;
      H[c * C * PC + e] = (c < nc) ? fld[c][q * PC + pl + P * r] : mk<R>(0, 0);
    }
  __shared__ NLArgs s_nl;
  const NLArgs &nl = s_nl;
  if (threadIdx.x == 0) s_nl = a.nl;
  __syncthreads();
  double t = a.t0;
  const double dt = nl.dt;
  c1_kinetic<R, N, TC>(cl, H, K, tw, kh, nc, a.s_f, a.s_b);
  t += 0.5 * dt;
  for (int j = 0; j < a.nk; j++) {
    if (threadIdx.x == 0) {
      s_nl.t1 = t + 0.5 * dt;
      s_nl.F = a.F ? a.F[j] : 1.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < C * PC; e += NT) {
      const int r = e / PC, pl = e % PC;
      const int i = q * PC + pl + P * r;
      const double x0 = (double)(i - nl.shift0) * nl.dx0;
      double om = 0, ec = 1, es = 0;
      if (nl.kind == K_BRAGG) bragg_coupling(nl, x0, om, ec, es);
      C_ v[MAXC];
      #pragma unroll
      for (int c = 0; c < TC; c++) v[c] = H[(c * C + r) * PC + pl];
      nl_point<R, TC>(nl, v, i, x0, om, ec, es);
      #pragma unroll
      for (int c = 0; c < TC; c++) H[(c * C + r) * PC + pl] = v[c];
    }
    __syncthreads();
    const bool last = (j == a.nk - 1);
    const double2 *tab[TC];
    #pragma unroll
    for (int c = 0; c < TC; c++) tab[c] = last ? kh[c] : kf[c];
    c1_kinetic<R, N, TC>(cl, H, K, tw, tab, nc, a.s_f, a.s_b);
    t += last ? 0.5 * dt : dt;
  }
  #pragma unroll
  for (int c = 0; c < TC; c++)
    if (c < nc)
      for (int e = threadIdx.x; e < C * PC; e += NT) {
        const int r = e / PC, pl = e % PC;
        fld[c][q * PC + pl + P * r] = H[c * C * PC + e];
      }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

}  // namespace atus

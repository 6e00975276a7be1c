// pass3.cuh -- register-staged passes for pencils of 512, 1024 and 2048 points.
//
// N = 16 M, M = 16 R3 (R3 = 2, 4, 8).  With n = t + M r (t < M, r < 16) and
// k = q + 16 k2:
//
//   X[q + 16 k2] = sum_t W_M^{t k2} W_N^{t q} sum_r x[t + M r] W_16^{r q}
//
// Stage 1: thread t of a pencil holds the 16 inputs t + M r, takes the radix-16
// DFT over r and the twiddles W_N^{t q}.  The M-point DFT over t is done in
// two more stages with t = j2 + R3 r2, k2 = q2 + 16 k3: stage 2 (thread
// (q, j2)) a radix-16 DFT over r2 of column q, times W_M^{j2 q2}; stage 3
// (thread (q, q2') with q2 = q2' + R3 s, s < 16 / R3) radix-R3 DFTs over j2.
// Two shared-memory exchanges per transform.  The thread t = q + 16 q2' ends
// with X[t + M (s + (16 / R3) k3)] -- again the inputs t + M r of a stage 1 --
// so FFT -> point-wise operator -> IFFT chains in registers, as in pass2.cuh.
//
// Exchange layouts (per pencil-component, complex values): after stage 1 row
// t, column q at 17 t + q; after stage 2 (q, j2, q2) at q + 16 (j2 + R3 q2).
// In both, the threads of a quarter warp (8 x 16-byte accesses) differ in the
// column q or the row t and hit distinct bank groups.
#pragma once
#include "pass2.cuh"

namespace atus {

template <typename R> struct Tile3;
template <> struct Tile3<double> { static constexpr int NT = 128; };
template <> struct Tile3<float> { static constexpr int NT = 256; };

// Strided tiles hold 8 adjacent pencils, so that a warp's loads cover
// 64-byte (complex64) or 128-byte (FP64) runs of a row; FP64 2048-point
// pencils take 4 (512 threads of 16 complex128 values fill the register
// file).  Measured on the 2048^2 complex64 x pass: 4 -> 8 pencils 0.072 ->
// 0.050 ms.
template <typename R, int N, int TC, bool STRIDED>
struct P3Cfg {
  static constexpr int M = N / 16;   // stage-1 butterflies: threads per pencil-component
  static constexpr int R3 = M / 16;  // radix of stage 3
  static constexpr int T3 = 16 / R3; // stage-3 butterflies per thread
  static constexpr int BMIN = STRIDED ? ((sizeof(R) == 8 && M * TC * 8 > 512) ? 4 : 8) : 1;
  static constexpr int NT_MIN = M * TC * BMIN;
  static constexpr int NT = (NT_MIN > Tile3<R>::NT) ? NT_MIN : Tile3<R>::NT;
  static constexpr int NPC = NT / M; // pencil-components per tile
  static constexpr int B = NPC / TC; // pencils per tile
  // Pencil pitch of the exchange rows.  A bank group (the threads whose
  // 128-byte wavefront is served at once: G = 8 complex128 or 16 complex64
  // values) holds, in strided tiles, B pencils x G / B consecutive t; pitch
  // PB = G / B (mod G) puts them on G distinct banks (the rows' own offsets
  // are t mod G, 17 M = 0 mod G).  Contiguous tiles: a group is one pencil.
  static constexpr int G = 128 / (int)sizeof(cplx<R>);
  static constexpr int PB = 17 * M + ((STRIDED && B < G) ? G / B : 1);
  static constexpr size_t smem_ex = sizeof(cplx<R>) * NPC * PB;
  // W_N^{t q} (row q, column t) and W_M^{j2 q2} (row q2, column j2)
  static constexpr int TWN_N = 16 * M, TWN_M = 16 * R3;
  static constexpr size_t smem = smem_ex + sizeof(typename TwTab<R>::type) * (TWN_N + TWN_M);
  // CTAs per SM the register budget is sized for: what shared memory allows,
  // at most 512 / NT (128 registers a thread)
  static constexpr int BY_SMEM = (int)((227 * 1024) / (smem + 1024));
  static constexpr int BY_REGS = 512 / NT;
  static constexpr int MINB = BY_SMEM < 1 ? 1 : (BY_SMEM < BY_REGS ? BY_SMEM : BY_REGS);
};

// One transform of the thread's 16 values v (inputs t + M r on entry, points
// t + M r on return).  ex: the pencil-component's exchange rows.
template <typename R, int N, int DIR>
__device__ __forceinline__ void p3_transform(cplx<R> *v, cplx<R> *ex, const typename TwTab<R>::type *twN,
                                             const typename TwTab<R>::type *twM, int t) {
  using C = cplx<R>;
  constexpr int M = N / 16, R3 = M / 16, T3 = 16 / R3;
  // stage 1: radix 16 over r, twiddles W_N^{t q}
  dft16<DIR>(v);
  #pragma unroll
  for (int q = 1; q < 16; q++) v[q] = twmul<DIR>(v[q], twN[q * M + t]);
  __syncthreads();
  #pragma unroll
  for (int q = 0; q < 16; q++) ex[17 * t + q] = v[q];
  __syncthreads();
  // stage 2: thread (qa, j2), radix 16 over r2 of column qa, rows j2 + R3 r2
  const int qa = t & 15, j2 = t >> 4;
  #pragma unroll
  for (int r2 = 0; r2 < 16; r2++) v[r2] = ex[17 * (j2 + R3 * r2) + qa];
  dft16<DIR>(v);
  #pragma unroll
  for (int q2 = 1; q2 < 16; q2++) v[q2] = twmul<DIR>(v[q2], twM[q2 * R3 + j2]);
  __syncthreads();
  #pragma unroll
  for (int q2 = 0; q2 < 16; q2++) ex[qa + 16 * (j2 + R3 * q2)] = v[q2];
  __syncthreads();
  // stage 3: thread (qa, q2p), butterflies q2 = q2p + R3 s, radix R3 over j2
  const int q2p = t >> 4;
  #pragma unroll
  for (int s = 0; s < T3; s++) {
    C u[R3];
    #pragma unroll
    for (int jj = 0; jj < R3; jj++) u[jj] = ex[qa + 16 * (jj + R3 * (q2p + R3 * s))];
    dftR<R3, DIR>(u);
    #pragma unroll
    for (int k3 = 0; k3 < R3; k3++) v[s + T3 * k3] = u[k3];
  }
}

template <typename R, int N, int TC, bool STRIDED>
__device__ __forceinline__ void p3_setup(const PassArgs &a, unsigned char *smem_raw) {
  using TW = typename TwTab<R>::type;
  using Cfg = P3Cfg<R, N, TC, STRIDED>;
  constexpr int M = Cfg::M, R3 = Cfg::R3;
  TW *const twN = reinterpret_cast<TW *>(smem_raw + Cfg::smem_ex);
  TW *const twM = twN + Cfg::TWN_N;
  const TW *tw = (const TW *)a.tw;
  for (int e = threadIdx.x; e < Cfg::TWN_N; e += Cfg::NT) {
    const int q = e / M, t = e % M;
    twN[e] = tw[(t * q) * (TWN / N)];
  }
  for (int e = threadIdx.x; e < Cfg::TWN_M; e += Cfg::NT) {
    const int q2 = e / R3, j2 = e % R3;
    twM[e] = tw[(j2 * q2) * (TWN / M)];
  }
}

// One work item: the tile g of the pass described by a (as p2_item).
template <typename R, int N, int TC, int MODE, bool STRIDED>
__device__ __forceinline__ void p3_item(const PassArgs &a, const TileGeo &g, unsigned char *smem_raw, double *s_om,
                                        double *s_ec, double *s_es) {
  using C = cplx<R>;
  using TW = typename TwTab<R>::type;
  using Cfg = P3Cfg<R, N, TC, STRIDED>;
  constexpr int M = Cfg::M, B = Cfg::B, NT = Cfg::NT, PB = Cfg::PB;
  static_assert(N >= 512 && N <= 2048, "three-stage pencils only");
  static_assert(Cfg::NPC * M == NT, "one thread per stage-1 butterfly");
  C *const ex = reinterpret_cast<C *>(smem_raw);
  const TW *const twN = reinterpret_cast<const TW *>(smem_raw + Cfg::smem_ex);
  const TW *const twM = twN + Cfg::TWN_N;
  const int tid = threadIdx.x;
  int b, t, c;
  if (STRIDED) { b = tid % B; t = (tid / B) % M; c = tid / (B * M); }
  else { t = tid % M; b = (tid / M) % B; c = tid / (M * B); }
  C *const my = ex + (c * B + b) * PB;
  const int nc = a.per_comp ? 1 : a.nc;
  const bool live = (b < g.nb) && (c < nc);
  C *const f = (C *)pick(a.psi, g.comp0 + c);
  const int64_t lb = g.base0 + b * g.pstride;  // grid index of the pencil's point 0
  const int64_t step = (int64_t)M * a.sa;      // distance of points t + M r and t + M (r+1)
  const C *src = live ? f + lb + (int64_t)t * a.sa : nullptr;

  if constexpr (MODE == M2_NL && TC > 1) {
    if (a.nl.kind == K_BRAGG && a.axis != 0)
      for (int p = tid; p < B; p += NT) {
        double om = 0, ec = 1, es = 0;
        if (p < g.nb) {
          int ix, iy, iz;
          idx3(a.g, g.base0 + p * g.pstride, ix, iy, iz);
          bragg_coupling(a.nl, (double)(ix - a.nl.shift0) * a.nl.dx0, om, ec, es);
        }
        s_om[p] = om; s_ec[p] = ec; s_es[p] = es;
      }
  }

  C v[16];
  #pragma unroll
  for (int r = 0; r < 16; r++) v[r] = live ? src[r * step] : mk<R>(0, 0);

  // one-component potential step: the potential of the thread's 16 points
  // is requested into L2 now and loaded eight points ahead of its use after
  // the inverse transform (behind the per-point branches each load would
  // wait on its own)
  const double *const Vp = a.nl.V[0];
  const bool preV = MODE == M2_NL && TC == 1 && a.nl.kind == K_NL && Vp != nullptr && live;
  if (preV) {
    #pragma unroll
    for (int m = 0; m < 16; m++)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(Vp + lb + (int64_t)(t + M * m) * a.sa));
  }

  if constexpr (MODE == M2_FWD) {
    p3_transform<R, N, -1>(v, my, twN, twM, t);
  } else if constexpr (MODE == M2_INV) {
    p3_transform<R, N, +1>(v, my, twN, twM, t);
  } else if constexpr (MODE == M2_KIN) {
    p3_transform<R, N, -1>(v, my, twN, twM, t);
    int p0[3];
    idx3(a.g, lb, p0[0], p0[1], p0[2]);
    if (a.op == OP_KIN) {
      // psi^ <- ((psi^ s_f) K) s_b in FP64 (complex64 fields: the scales
      // folded into K), K = K_along x the product of the other axis factors
      const double2 *kx = a.kt[0][0], *ky = a.kt[0][1], *kz = a.kt[0][2];
      #pragma unroll
      for (int cc = 1; cc < MAXC; cc++)
        if (g.comp0 == cc) { kx = a.kt[cc][0]; ky = a.kt[cc][1]; kz = a.kt[cc][2]; }
      const double2 KX = __ldg(&kx[p0[0]]), KY = __ldg(&ky[p0[1]]), KZ = __ldg(&kz[p0[2]]);
      double2 Kp = (a.axis == 0) ? cmul(KY, KZ) : (a.axis == 1) ? cmul(KX, KZ) : cmul(KX, KY);
      const double2 *along = (a.axis == 0) ? kx : (a.axis == 1) ? ky : kz;
      if (sizeof(R) == 4) {
        const double sc = a.s_f * a.s_b;
        Kp.x *= sc;
        Kp.y *= sc;
      }
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        const int i = t + M * m;
        const double2 K = cmul(__ldg(&along[i]), Kp);
        double2 u = to_d<R>(v[m]);
        if (sizeof(R) == 8) {
          u.x *= a.s_f;
          u.y *= a.s_f;
        }
        u = cmul(u, K);
        if (sizeof(R) == 8) {
          u.x *= a.s_b;
          u.y *= a.s_b;
        }
        v[m] = from_d<R>(u);
      }
    } else if (a.op == OP_FILT) {
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        const int i = t + M * m;
        double phi = 0;
        #pragma unroll
        for (int ax = 0; ax < 3; ax++) {
          const int ii = (ax == a.axis) ? i : p0[ax];
          const int tt = (ii + a.n[ax] / 2) % a.n[ax];
          const double k = a.dk[ax] * (double)(tt - a.n[ax] / 2);
          phi += (k * a.filt_alpha) * k;
        }
        const double fk = (a.filt_mode == FILT_SOBOLEV ? 1.0 / (1.0 + phi) : -phi) * a.filt_scale;
        v[m].x = (R)((double)v[m].x * fk);
        v[m].y = (R)((double)v[m].y * fk);
      }
    }
    p3_transform<R, N, +1>(v, my, twN, twM, t);
  } else {  // M2_NL: IFFT -> potential step -> FFT
    p3_transform<R, N, +1>(v, my, twN, twM, t);
    if constexpr (TC == 1) {
      int p0[3];
      idx3(a.g, lb, p0[0], p0[1], p0[2]);
      constexpr int AHEAD = 8;  // potential loads in flight
      double vpre[16];
      auto load_v = [&](int m) { vpre[m] = preV ? __ldg(&Vp[lb + (int64_t)(t + M * m) * a.sa]) : 0.0; };
      #pragma unroll
      for (int m = 0; m < AHEAD; m++) load_v(m);
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        if (m + AHEAD < 16) load_v(m + AHEAD);
        const int i = t + M * m;
        const int64_t l = lb + (int64_t)i * a.sa;
        const int ix = (a.axis == 0) ? i : p0[0];
        const double x0 = (double)(ix - a.nl.shift0) * a.nl.dx0;
        double om = 0, ec = 1, es = 0;
        if (a.nl.kind == K_BRAGG) bragg_coupling(a.nl, x0, om, ec, es);
        C u[MAXC];
        u[0] = v[m];
        if (live) nl_point<R, TC, true>(a.nl, u, l, x0, om, ec, es, vpre[m]);
        v[m] = u[0];
      }
    } else {
      // all components of a point meet in shared memory (natural order)
      __syncthreads();
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        const int i = t + M * m;
        my[ex_at(i >> 4, i & 15)] = v[m];
      }
      __syncthreads();
      constexpr int PPT = 16 / TC;  // points per thread
      const bool bragg = (a.nl.kind == K_BRAGG);
      #pragma unroll 1
      for (int u_ = 0; u_ < PPT; u_++) {
        const int p = tid + NT * u_;
        int pb, i;
        if (STRIDED) { pb = p % B; i = p / B; } else { i = p % N; pb = p / N; }
        if (pb < g.nb) {
          const int64_t l = g.base0 + pb * g.pstride + (int64_t)i * a.sa;
          int ix, iy, iz;
          idx3(a.g, l, ix, iy, iz);
          const double x0 = (double)(ix - a.nl.shift0) * a.nl.dx0;
          double om = 0, ec = 1, es = 0;
          if (bragg) {
            if (a.axis == 0) bragg_coupling(a.nl, x0, om, ec, es);
            else { om = s_om[pb]; ec = s_ec[pb]; es = s_es[pb]; }
          }
          C u[MAXC];
          #pragma unroll
          for (int cc = 0; cc < TC; cc++) u[cc] = ex[(cc * B + pb) * PB + ex_at(i >> 4, i & 15)];
          nl_point<R, TC>(a.nl, u, l, x0, om, ec, es);
          #pragma unroll
          for (int cc = 0; cc < TC; cc++) ex[(cc * B + pb) * PB + ex_at(i >> 4, i & 15)] = u[cc];
        }
      }
      __syncthreads();
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        const int i = t + M * m;
        v[m] = my[ex_at(i >> 4, i & 15)];
      }
    }
    p3_transform<R, N, -1>(v, my, twN, twM, t);
  }

  if (live) {
    C *dst = f + lb + (int64_t)t * a.sa;
    #pragma unroll
    for (int m = 0; m < 16; m++) dst[m * step] = v[m];
  }
}

// Strided tiles: the CTA's next tile requested into L2 while this one is
// transformed (one prefetch per 128-byte line).
template <typename R, int N, int B>
__device__ __forceinline__ void p3_prefetch_l2(const PassArgs &a, const TileGeo &g, int nt) {
  constexpr int LINE = 128 / (int)sizeof(cplx<R>);
  constexpr int SEG = (B + LINE - 1) / LINE;
  const int nc = a.per_comp ? 1 : a.nc;
  for (int e = threadIdx.x; e < nc * N * SEG; e += nt) {
    const int c = e / (N * SEG), rem = e % (N * SEG);
    const int i = rem / SEG, seg = rem % SEG;
    if (seg * LINE >= g.nb) continue;
    const cplx<R> *f = (const cplx<R> *)pick(a.psi, g.comp0 + c);
    const cplx<R> *p = f + g.base0 + (int64_t)(seg * LINE) * g.pstride + (int64_t)i * a.sa;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

template <typename R, int N, int TC, int MODE, bool STRIDED>
__global__ void __launch_bounds__(P3Cfg<R, N, TC, STRIDED>::NT, P3Cfg<R, N, TC, STRIDED>::MINB)
    pass3_kernel(PassArgs a) {
  using Cfg = P3Cfg<R, N, TC, STRIDED>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_om[Cfg::B], s_ec[Cfg::B], s_es[Cfg::B];
  p3_setup<R, N, TC, STRIDED>(a, smem_raw);
  __syncthreads();  // twiddle rows visible to every warp
  const int64_t W = a.per_comp ? a.ntiles * a.ncomp_grid : a.ntiles;
  for (int64_t w = blockIdx.x; w < W; w += gridDim.x) {
    if (STRIDED && w + gridDim.x < W) p3_prefetch_l2<R, N, Cfg::B>(a, tile_geo<Cfg::B, N>(a, w + gridDim.x), Cfg::NT);
    p3_item<R, N, TC, MODE, STRIDED>(a, tile_geo<Cfg::B, N>(a, w), smem_raw, s_om, s_ec, s_es);
  }
}

}  // namespace atus

// pass2.cuh -- register-staged pass kernel for pencils of 32..256 points.
//
// A pencil of N = 16 R2 points is transformed in the two Stockham stages of
// fft_tile (radix 16 over inputs j + R2 r, then radix R2 with twiddles
// exp(-+2 pi i r k / N)), with the same arithmetic in the same order.  What
// differs is where the data lives between the stages:
//
//   HBM -> registers (stage-1 inputs)  -> stage 1 -> shared exchange ->
//   stage 2 -> registers (outputs j + R2 m, m < 16) -> HBM
//
// The thread that reads inputs j + R2 r (r < 16) of stage 1 ends up with the
// outputs j + R2 m of stage 2, which are again the inputs of a stage 1.  So
// FFT -> point-wise operator -> IFFT runs in registers with one shared-memory
// exchange per transform, where the tile kernel (pass_kernel) makes six sweeps
// through shared memory per transform plus the tile load and store.  Twiddles
// come from a padded per-pencil-length table in shared memory.
//
// Thread layout: along a strided axis consecutive threads take consecutive
// pencils (the inner grid index), so one warp-wide load covers whole 128-byte
// rows; along the contiguous axis consecutive threads take consecutive points.
#pragma once
#include "kernels.cuh"

namespace atus {

// Tile budget (complex values) and threads; one thread owns 16 values.
template <typename R> struct Tile2;
template <> struct Tile2<double> { static constexpr int E = 2048, NT = 128, MINB = 5; };
template <> struct Tile2<float> { static constexpr int E = 4096, NT = 256, MINB = 3; };

template <typename R, int N, int TC>
struct P2Cfg {
  static constexpr int R2 = N / 16;        // stage-2 radix
  static constexpr int T2 = 16 / R2;       // stage-2 butterflies per thread
  static constexpr int E = Tile2<R>::E;
  static constexpr int NT = Tile2<R>::NT;
  static constexpr int B = E / (N * TC);   // pencils per tile
  static constexpr int NPC = B * TC;       // pencil-components per tile
  static constexpr int PB = 17 * R2 + 1;   // exchange pitch: R2 rows of 16 + 1 pad, odd
  static constexpr int TP = R2 + 1;        // twiddle row pitch (odd)
  static constexpr int TWP = 16 * TP;      // twiddle table: row k holds W_N^{r k}, r < R2
  static constexpr size_t smem_ex = sizeof(cplx<R>) * NPC * PB;
  static constexpr size_t smem_tw = sizeof(typename TwTab<R>::type) * TWP;
  static constexpr size_t smem = smem_ex + smem_tw;
  // k-space passes also keep the along-axis kinetic factors of up to two
  // components in shared memory (FP64)
  static constexpr size_t smem_kin = smem + 2 * N * sizeof(double2);
  // the kinetic factors go to shared memory only if that keeps MINB CTAs per SM
  static constexpr bool kin_smem = (smem_kin + 1024) * Tile2<R>::MINB <= 228 * 1024;
};

// Exchange layout of one pencil-component: row-major R2 x 16 with row pitch
// 17.  Stage-1 butterfly j writes row j (its 16 outputs, Stockham index
// 16 j + q); stage-2 butterfly k reads column k.  Point i of the natural order
// sits at row i / 16, column i % 16.
__device__ __forceinline__ int ex_at(int row, int col) { return 17 * row + col; }

// Stage 2 of a transform: butterflies k = j + R2 t (t < T2) of the pencil whose
// exchange rows start at ex; o[t + T2 r] = output k + 16 r = point j + R2 (t + T2 r).
// Twiddle W_N^{r k} is entry r of row k (pitch R2 + 1, odd): the eight threads
// of a quarter warp, which hold eight different k on the contiguous axis, hit
// eight different bank groups.
template <typename R, int N, int DIR>
__device__ __forceinline__ void p2_stage2(const cplx<R> *ex, const typename TwTab<R>::type *twS, int j, cplx<R> *o) {
  using C = cplx<R>;
  constexpr int R2 = N / 16, T2 = 16 / R2;
  #pragma unroll
  for (int t = 0; t < T2; t++) {
    const int k = j + R2 * t;
    C u[R2];
    #pragma unroll
    for (int r = 0; r < R2; r++) u[r] = ex[ex_at(r, k)];
    #pragma unroll
    for (int r = 1; r < R2; r++) u[r] = twmul<DIR>(u[r], twS[k * (R2 + 1) + r]);
    dftR<R2, DIR>(u);
    #pragma unroll
    for (int r = 0; r < R2; r++) o[t + T2 * r] = u[r];
  }
}

// One transform of the thread's 16 values v (stage-1 inputs j + R2 r on entry,
// points j + R2 m on return).  The leading barrier protects the exchange rows
// that other threads may still be reading from the previous use.  WARP: the
// R2 threads of each pencil are consecutive lanes of one warp (the contiguous
// mapping), so the exchange needs only a warp barrier; the strided mapping
// spreads a pencil over the CTA's warps and needs the CTA barrier.
template <typename R, int N, int DIR, bool WARP = false>
__device__ __forceinline__ void p2_transform(cplx<R> *v, cplx<R> *ex, const typename TwTab<R>::type *twS, int j) {
  dft16<DIR>(v);
  if constexpr (WARP) __syncwarp(); else __syncthreads();
  #pragma unroll
  for (int q = 0; q < 16; q++) ex[ex_at(j, q)] = v[q];
  if constexpr (WARP) __syncwarp(); else __syncthreads();
  p2_stage2<R, N, DIR>(ex, twS, j, v);
}

// Shared-memory set-up of a CTA, once per launch: the twiddle rows and, for
// k-space passes, the along-axis kinetic factors of components 0 and 1.
// Returns whether those factors are in shared memory.
template <typename R, int N, int TC, int MODE>
__device__ __forceinline__ bool p2_setup(const PassArgs &a, unsigned char *smem_raw) {
  using TW = typename TwTab<R>::type;
  using Cfg = P2Cfg<R, N, TC>;
  constexpr int R2 = Cfg::R2, NT = Cfg::NT;
  const int tid = threadIdx.x;
  TW *const twS = reinterpret_cast<TW *>(smem_raw + Cfg::smem_ex);
  {  // W_N^{r k} = exp(-2 pi i r k / N) from the TWN-point table
    const TW *tw = (const TW *)a.tw;
    for (int e = tid; e < 16 * R2; e += NT) {
      const int k = e / R2, r = e % R2;
      twS[k * Cfg::TP + r] = tw[(r * k) * (TWN / N)];
    }
  }
  // k-space passes: along-axis kinetic factors of components 0 and 1
  double2 *const s_kt = reinterpret_cast<double2 *>(smem_raw + Cfg::smem);
  const bool kt_shared = (MODE == M2_KIN || MODE == M2_KIN_RABI) && Cfg::kin_smem && a.op == OP_KIN && a.ncomp_grid <= 2;
  if (kt_shared) {
    for (int e = tid; e < a.ncomp_grid * N; e += NT) {
      const int cc = e / N, i = e % N;
      const double2 *t0 = (a.axis == 0) ? a.kt[0][0] : (a.axis == 1) ? a.kt[0][1] : a.kt[0][2];
      const double2 *t1 = (a.axis == 0) ? a.kt[1][0] : (a.axis == 1) ? a.kt[1][1] : a.kt[1][2];
      s_kt[e] = (cc == 0) ? t0[i] : t1[i];
    }
  }
  return kt_shared;
}

// One work item: the tile g of the pass described by a.
// Rabi sums of one thread's 16 values (k-space points j + R2 m of the pencil
// whose point 0 has axis indices p0) into rq, with the ball rule of
// compute_rabi_integrals (include/CRT_Base_IF.h:231-257): a point inside a
// ball adds to the current bin and the bin index does not advance for it.
template <typename R, int N>
__device__ __forceinline__ void p2_rabi(const PassArgs &a, int ci, const int *p0, int j, const cplx<R> *v, double *rq) {
  constexpr int R2 = N / 16;
  #pragma unroll 1
  for (int m = 0; m < 16; m++) {
    const int i = j + R2 * m;
    const double den = (double)v[m].x * (double)v[m].x + (double)v[m].y * (double)v[m].y;
    double k[3];
    #pragma unroll
    for (int ax = 0; ax < 3; ax++) {
      const int idx = (ax == a.axis) ? i : p0[ax];
      const int sh = a.n[ax] / 2;
      const int t = (idx + sh) % a.n[ax];
      k[ax] = a.dk[ax] * (double)(t - sh);
    }
    int jb = 0;
    for (int q = 0; q < a.rabi_n; q++) {
      double dd = 0;
      #pragma unroll
      for (int ax = 0; ax < 3; ax++) {
        const double d = a.rabi_k0[ci * a.rabi_n + q][ax] - k[ax];
        dd += d * d;
      }
      if (sqrt(dd) < a.rabi_thr) {
        rq[ci * a.rabi_n + jb] += den;
        continue;
      }
      jb++;
    }
  }
}

// After-load hook of p2_item (the TMA kernel refills the tile buffer there).
struct P2NoHook {
  __device__ __forceinline__ void operator()() const {}
};

// Tile of a strided pass as a TMA box writes it: row i (point i of the B
// pencils) is B values.  Rows of 128 bytes come with the 128-byte swizzle
// (16-byte chunk c at position c ^ (i & 7)); longer rows unswizzled (the
// threads of a quarter warp read consecutive pencils of one row).  Value of
// pencil b at point i.
template <typename R, int B>
__device__ __forceinline__ cplx<R> p2_tile_at(const unsigned char *tile, int i, int b) {
  constexpr int ROW = B * (int)sizeof(cplx<R>);
  if constexpr (ROW != 128)
    return *reinterpret_cast<const cplx<R> *>(tile + i * ROW + b * (int)sizeof(cplx<R>));
  else if constexpr (sizeof(R) == 8)
    return *reinterpret_cast<const cplx<R> *>(tile + i * 128 + ((b ^ (i & 7)) << 4));
  else
    return *reinterpret_cast<const cplx<R> *>(tile + i * 128 + (((b >> 1) ^ (i & 7)) << 4) + ((b & 1) << 3));
}

// One work item.  SMEM_TILE (strided passes): the tile's inputs come from
// `tile` (swizzled, see p2_tile_at) instead of global memory, and hook()
// runs once every thread has taken its values.
template <typename R, int N, int TC, int MODE, bool STRIDED, bool SMEM_TILE = false, typename Hook = P2NoHook>
__device__ __forceinline__ void p2_item(const PassArgs &a, const TileGeo &g, unsigned char *smem_raw, bool kt_shared,
                                        double *s_om, double *s_ec, double *s_es, double *rq = nullptr,
                                        const unsigned char *tile = nullptr, Hook hook = Hook()) {
  using C = cplx<R>;
  using TW = typename TwTab<R>::type;
  using Cfg = P2Cfg<R, N, TC>;
  constexpr int R2 = Cfg::R2, B = Cfg::B, NT = Cfg::NT, PB = Cfg::PB;
  static_assert(N >= 32 && N <= 256, "two-stage pencils only");
  static_assert(Cfg::NPC * R2 == NT, "one thread per stage-1 butterfly");
  C *const ex = reinterpret_cast<C *>(smem_raw);
  const TW *const twS = reinterpret_cast<const TW *>(smem_raw + Cfg::smem_ex);
  const double2 *const s_kt = reinterpret_cast<const double2 *>(smem_raw + Cfg::smem);
  const int tid = threadIdx.x;
  int b, j, c;
  if (STRIDED) { b = tid % B; j = (tid / B) % R2; c = tid / (B * R2); }
  else { j = tid % R2; b = (tid / R2) % B; c = tid / (R2 * B); }
  C *const my = ex + (c * B + b) * PB;
  const int nc = a.per_comp ? 1 : a.nc;
  const bool live = (b < g.nb) && (c < nc);
  C *const f = (C *)pick(a.psi, g.comp0 + c);
  const int64_t lb = g.base0 + b * g.pstride;  // grid index of the pencil's point 0
  const int64_t step = (int64_t)R2 * a.sa;     // distance of points j + R2 m and j + R2 (m+1)
  const C *src = live ? f + lb + (int64_t)j * a.sa : nullptr;

  if constexpr (MODE == M2_NL && TC > 1) {
    // coupling of each pencil (x is constant along it); read after the
    // barriers of the first transform
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
  if constexpr (SMEM_TILE) {
    static_assert(STRIDED, "shared-memory tiles of strided passes only");
    #pragma unroll
    for (int r = 0; r < 16; r++) v[r] = p2_tile_at<R, B>(tile, j + R2 * r, b);
    hook();
  } else {
    #pragma unroll
    for (int r = 0; r < 16; r++) v[r] = live ? src[r * step] : mk<R>(0, 0);
  }

  if constexpr (MODE == M2_FWD) {
    p2_transform<R, N, -1, !STRIDED>(v, my, twS, j);
  } else if constexpr (MODE == M2_INV) {
    p2_transform<R, N, +1, !STRIDED>(v, my, twS, j);
  } else if constexpr (MODE == M2_KIN || MODE == M2_KIN_RABI) {
    p2_transform<R, N, -1, !STRIDED>(v, my, twS, j);
    int p0[3];
    idx3(a.g, lb, p0[0], p0[1], p0[2]);
    if constexpr (MODE == M2_KIN_RABI) {
      int ci = -1;
      for (int c = 0; c < a.rabi_ncomp; c++)
        if (a.rabi_comp[c] == g.comp0) ci = c;
      if (live && ci >= 0) p2_rabi<R, N>(a, ci, p0, j, v, rq);
    }
    if (a.op == OP_KIN) {
      // psi^ <- ((psi^ s_f) K) s_b in FP64, K = K_along (product of the other
      // two axis factors, x before y before z); complex64 fields take the
      // scales folded into K
      const double2 *kx = a.kt[0][0], *ky = a.kt[0][1], *kz = a.kt[0][2];
      #pragma unroll
      for (int cc = 1; cc < MAXC; cc++)
        if (g.comp0 == cc) { kx = a.kt[cc][0]; ky = a.kt[cc][1]; kz = a.kt[cc][2]; }
      const double2 KX = __ldg(&kx[p0[0]]), KY = __ldg(&ky[p0[1]]), KZ = __ldg(&kz[p0[2]]);
      double2 Kp = (a.axis == 0) ? cmul(KY, KZ) : (a.axis == 1) ? cmul(KX, KZ) : cmul(KX, KY);
      const double2 *along = (a.axis == 0) ? kx : (a.axis == 1) ? ky : kz;
      const double2 *sk = s_kt + (g.comp0 == 1 ? N : 0);
      if (sizeof(R) == 4) {
        const double sc = a.s_f * a.s_b;
        Kp.x *= sc;
        Kp.y *= sc;
      }
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        const int i = j + R2 * m;
        const double2 K = cmul(kt_shared ? sk[i] : __ldg(&along[i]), Kp);
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
        const int i = j + R2 * m;
        double phi = 0;
        #pragma unroll
        for (int ax = 0; ax < 3; ax++) {
          const int ii = (ax == a.axis) ? i : p0[ax];
          const int t = (ii + a.n[ax] / 2) % a.n[ax];
          const double k = a.dk[ax] * (double)(t - a.n[ax] / 2);
          phi += (k * a.filt_alpha) * k;
        }
        const double fk = (a.filt_mode == FILT_SOBOLEV ? 1.0 / (1.0 + phi) : -phi) * a.filt_scale;
        v[m].x = (R)((double)v[m].x * fk);
        v[m].y = (R)((double)v[m].y * fk);
      }
    }
    p2_transform<R, N, +1, !STRIDED>(v, my, twS, j);
  } else {  // M2_NL: IFFT -> potential step -> FFT
    p2_transform<R, N, +1, !STRIDED>(v, my, twS, j);
    if constexpr (TC == 1) {
      int p0[3];
      idx3(a.g, lb, p0[0], p0[1], p0[2]);
      // the potential, loaded four points ahead of its use (behind the
      // per-point branches each load would wait on its own)
      const double *const Vp = a.nl.V[0];
      const bool preV = a.nl.kind == K_NL && Vp != nullptr && live;
      constexpr int AHEAD = 4;
      double vpre[16];
      auto load_v = [&](int m) { vpre[m] = preV ? __ldg(&Vp[lb + (int64_t)(j + R2 * m) * a.sa]) : 0.0; };
      #pragma unroll
      for (int m = 0; m < AHEAD; m++) load_v(m);
      #pragma unroll
      for (int m = 0; m < 16; m++) {
        if (m + AHEAD < 16) load_v(m + AHEAD);
        const int i = j + R2 * m;
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
        const int i = j + R2 * m;
        my[ex_at(i >> 4, i & 15)] = v[m];
      }
      __syncthreads();
      constexpr int PPT = 16 / TC;  // points per thread
      const bool bragg = (a.nl.kind == K_BRAGG);
      #pragma unroll 1  // measured fastest: unrolling 2/4/8 points was 4-50 % slower
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
      for (int r = 0; r < 16; r++) {
        const int i = j + R2 * r;
        v[r] = my[ex_at(i >> 4, i & 15)];
      }
    }
    p2_transform<R, N, -1, !STRIDED>(v, my, twS, j);
  }

  if (live) {
    C *dst = f + lb + (int64_t)j * a.sa;
    #pragma unroll
    for (int m = 0; m < 16; m++) dst[m * step] = v[m];
  }
}

// Strided tiles: asks L2 for the CTA's next tile (one prefetch per 128-byte
// line; the B pencils of a row are adjacent, the N rows sa apart) while this
// one is transformed, so that its loads wait on L2 rather than HBM.  (The
// same for contiguous tiles measured slower.)
template <typename R, int N, int TC>
__device__ __forceinline__ void p2_prefetch_l2(const PassArgs &a, const TileGeo &g) {
  using Cfg = P2Cfg<R, N, TC>;
  constexpr int LINE = 128 / (int)sizeof(cplx<R>);  // complex values per 128-byte line
  constexpr int SEG = (Cfg::B + LINE - 1) / LINE;
  const int nc = a.per_comp ? 1 : a.nc;
  for (int e = threadIdx.x; e < nc * N * SEG; e += Cfg::NT) {
    const int c = e / (N * SEG), rem = e % (N * SEG);
    const int i = rem / SEG, seg = rem % SEG;
    if (seg * LINE >= g.nb) continue;
    const cplx<R> *f = (const cplx<R> *)pick(a.psi, g.comp0 + c);
    const cplx<R> *p = f + g.base0 + (int64_t)(seg * LINE) * g.pstride + (int64_t)i * a.sa;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

template <typename R, int N, int TC, int MODE, bool STRIDED>
__global__ void __launch_bounds__(Tile2<R>::NT, Tile2<R>::MINB) pass2_kernel(PassArgs a) {
  using Cfg = P2Cfg<R, N, TC>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double s_om[Cfg::B], s_ec[Cfg::B], s_es[Cfg::B];
  const bool kt_shared = p2_setup<R, N, TC, MODE>(a, smem_raw);
  __syncthreads();  // twiddle rows and kinetic factors visible to every warp
  const int64_t W = a.per_comp ? a.ntiles * a.ncomp_grid : a.ntiles;
  double rq[MODE == M2_KIN_RABI ? RED_MAXQ : 1];
  #pragma unroll
  for (int q = 0; q < (MODE == M2_KIN_RABI ? RED_MAXQ : 1); q++) rq[q] = 0.0;
  for (int64_t w = blockIdx.x; w < W; w += gridDim.x) {
    if (STRIDED && w + gridDim.x < W) p2_prefetch_l2<R, N, TC>(a, tile_geo<Cfg::B, N>(a, w + gridDim.x));
    p2_item<R, N, TC, MODE, STRIDED>(a, tile_geo<Cfg::B, N>(a, w), smem_raw, kt_shared, s_om, s_ec, s_es, rq);
  }
  if constexpr (MODE == M2_KIN_RABI) {
    // per-CTA sums in a fixed tree (the tiles of a CTA are fixed by the grid
    // size, so the result does not depend on scheduling)
    __syncthreads();
    double *sh = reinterpret_cast<double *>(smem_raw);
    for (int q = 0; q < a.rabi_ncomp * a.rabi_n; q++) {
      sh[threadIdx.x] = rq[q];
      __syncthreads();
      for (int s = Cfg::NT / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
      }
      if (threadIdx.x == 0) a.rabi_partial[blockIdx.x * RED_MAXQ + q] = sh[0];
      __syncthreads();
    }
  }
}

}  // namespace atus

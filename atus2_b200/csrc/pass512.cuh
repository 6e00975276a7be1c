// pass512.cuh -- register-staged passes for pencils of 512 complex64 points.
//
// The two-stage scheme of pass2.cuh with 512 = 16 x 32: stage 1 is radix 16
// over inputs j' + 32 r (j' < 32), stage 2 radix 32 over the exchange columns
// with twiddles exp(-+2 pi i r k / 512) -- a Stockham 16 x 32 transform.
// Each of the 16 threads of a pencil owns the 32 points j + 16 m: the inputs
// of stage-1 butterflies j and j + 16 (even and odd m) and the outputs of
// stage-2 butterfly j, so FFT -> operator -> IFFT again chains in registers
// with one shared-memory exchange per transform.  32 complex64 values are 64
// registers; complex128 would need twice that, so only FP32 fields use it.
#pragma once
#include "pass2.cuh"

namespace atus {

template <typename R, int TC>
struct P5Cfg {
  static constexpr int N = 512;
  static constexpr int E = 4096;             // complex values per tile
  static constexpr int VPT = 32;             // values per thread
  static constexpr int NT = E / VPT;         // 128 threads
  static constexpr int B = E / (N * TC);     // pencils per tile
  static constexpr int NPC = B * TC;
  // exchange pitch in 8-byte values, = 2 mod 16: in the strided layout the
  // 16 lanes of a half warp are 8 pencils b x 2 rows j, at b * PB + j (mod 16)
  // -- distinct; in the contiguous layout they are 16 columns of one pencil
  static constexpr int PB = 17 * 32 + 2;
  static constexpr int TP = 33;              // twiddle row pitch
  static constexpr size_t smem_ex = sizeof(cplx<R>) * NPC * PB;
  static constexpr size_t smem = smem_ex + sizeof(typename TwTab<R>::type) * 16 * TP;
};

// cos and sin of pi k / 16, k < 16 (exp(i 2 pi k / 32)).
__device__ __forceinline__ void cs32(int k, double &c, double &s) {
  constexpr double C8[9] = {1.0,
                            0.98078528040323044913,
                            0.92387953251128675613,
                            0.83146961230254523708,
                            0.70710678118654752440,
                            0.55557023301960222474,
                            0.38268343236508977173,
                            0.19509032201612826785,
                            0.0};
  if (k <= 8) {
    c = C8[k];
    s = C8[8 - k];
  } else {  // pi (8 + m) / 16: cos = -sin(pi m / 16), sin = cos(pi m / 16)
    c = -C8[16 - k];
    s = C8[k - 8];
  }
}

// 32-point DFT (direction DIR) as two 16-point DFTs of the even and odd
// samples: X[k] = E[k] + W^k O[k], X[k + 16] = E[k] - W^k O[k], W = e^{DIR 2 pi i/32}.
template <int DIR, typename C>
__device__ __forceinline__ void dft32(C *v) {
  C e[16], o[16];
  #pragma unroll
  for (int r = 0; r < 16; r++) {
    e[r] = v[2 * r];
    o[r] = v[2 * r + 1];
  }
  dft16<DIR>(e);
  dft16<DIR>(o);
  v[0] = cadd(e[0], o[0]);
  v[16] = csub(e[0], o[0]);
  #pragma unroll
  for (int k = 1; k < 16; k++) {
    double c, s;
    cs32(k, c, s);
    const double ds = DIR * s;
    C t;
    t.x = kmul(o[k].x, c) - kmul(o[k].y, ds);
    t.y = kmul(o[k].y, c) + kmul(o[k].x, ds);
    v[k] = cadd(e[k], t);
    v[k + 16] = csub(e[k], t);
  }
}

// One transform of the thread's 32 values (inputs j + 16 m on entry, points
// j + 16 m on return).
template <typename R, int DIR>
__device__ __forceinline__ void p5_transform(cplx<R> *v, cplx<R> *ex, const typename TwTab<R>::type *twS, int j) {
  using C = cplx<R>;
  C e[16], o[16];
  #pragma unroll
  for (int r = 0; r < 16; r++) {
    e[r] = v[2 * r];      // point j + 32 r: butterfly j
    o[r] = v[2 * r + 1];  // point j + 16 + 32 r: butterfly j + 16
  }
  dft16<DIR>(e);
  dft16<DIR>(o);
  __syncthreads();
  #pragma unroll
  for (int q = 0; q < 16; q++) {
    ex[ex_at(j, q)] = e[q];
    ex[ex_at(j + 16, q)] = o[q];
  }
  __syncthreads();
  #pragma unroll
  for (int r = 0; r < 32; r++) v[r] = ex[ex_at(r, j)];
  #pragma unroll
  for (int r = 1; r < 32; r++) v[r] = twmul<DIR>(v[r], twS[j * 33 + r]);
  dft32<DIR>(v);
}

template <typename R, int TC>
__device__ __forceinline__ void p5_setup(const PassArgs &a, unsigned char *smem_raw) {
  using TW = typename TwTab<R>::type;
  using Cfg = P5Cfg<R, TC>;
  TW *const twS = reinterpret_cast<TW *>(smem_raw + Cfg::smem_ex);
  const TW *tw = (const TW *)a.tw;
  for (int e = threadIdx.x; e < 16 * 32; e += Cfg::NT) {
    const int k = e / 32, r = e % 32;
    twS[k * Cfg::TP + r] = tw[(r * k) * (TWN / 512)];
  }
}

// One work item (tile g) of a pass over 512-point pencils; as p2_item.
template <typename R, int TC, int MODE, bool STRIDED>
__device__ __forceinline__ void p5_item(const PassArgs &a, const TileGeo &g, unsigned char *smem_raw, double *s_om,
                                        double *s_ec, double *s_es) {
  using C = cplx<R>;
  using TW = typename TwTab<R>::type;
  using Cfg = P5Cfg<R, TC>;
  constexpr int N = 512, B = Cfg::B, NT = Cfg::NT, PB = Cfg::PB;
  static_assert(Cfg::NPC * 16 == NT, "16 threads per pencil-component");
  C *const ex = reinterpret_cast<C *>(smem_raw);
  const TW *const twS = reinterpret_cast<const TW *>(smem_raw + Cfg::smem_ex);
  const int tid = threadIdx.x;
  int b, j, c;
  if (STRIDED) { b = tid % B; j = (tid / B) % 16; c = tid / (B * 16); }
  else { j = tid % 16; b = (tid / 16) % B; c = tid / (16 * B); }
  C *const my = ex + (c * B + b) * PB;
  const int nc = a.per_comp ? 1 : a.nc;
  const bool live = (b < g.nb) && (c < nc);
  C *const f = (C *)pick(a.psi, g.comp0 + c);
  const int64_t lb = g.base0 + b * g.pstride;
  const int64_t step = (int64_t)16 * a.sa;  // points j + 16 m and j + 16 (m + 1)
  const C *src = live ? f + lb + (int64_t)j * a.sa : nullptr;

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

  C v[32];
  #pragma unroll
  for (int m = 0; m < 32; m++) v[m] = live ? src[m * step] : mk<R>(0, 0);

  if constexpr (MODE == M2_FWD) {
    p5_transform<R, -1>(v, my, twS, j);
  } else if constexpr (MODE == M2_INV) {
    p5_transform<R, +1>(v, my, twS, j);
  } else if constexpr (MODE == M2_KIN) {
    p5_transform<R, -1>(v, my, twS, j);
    int p0[3];
    idx3(a.g, lb, p0[0], p0[1], p0[2]);
    const double2 *kx = a.kt[0][0], *ky = a.kt[0][1], *kz = a.kt[0][2];
    #pragma unroll
    for (int cc = 1; cc < MAXC; cc++)
      if (g.comp0 == cc) { kx = a.kt[cc][0]; ky = a.kt[cc][1]; kz = a.kt[cc][2]; }
    const double2 KX = __ldg(&kx[p0[0]]), KY = __ldg(&ky[p0[1]]), KZ = __ldg(&kz[p0[2]]);
    double2 Kp = (a.axis == 0) ? cmul(KY, KZ) : (a.axis == 1) ? cmul(KX, KZ) : cmul(KX, KY);
    const double2 *along = (a.axis == 0) ? kx : (a.axis == 1) ? ky : kz;
    const double sc = a.s_f * a.s_b;  // complex64 fields: the scales folded into K
    Kp.x *= sc;
    Kp.y *= sc;
    #pragma unroll
    for (int m = 0; m < 32; m++) {
      const double2 K = cmul(__ldg(&along[j + 16 * m]), Kp);
      v[m] = from_d<R>(cmul(to_d<R>(v[m]), K));
    }
    p5_transform<R, +1>(v, my, twS, j);
  } else {  // M2_NL
    p5_transform<R, +1>(v, my, twS, j);
    if constexpr (TC == 1) {
      int p0[3];
      idx3(a.g, lb, p0[0], p0[1], p0[2]);
      #pragma unroll 4
      for (int m = 0; m < 32; m++) {
        const int i = j + 16 * m;
        const int64_t l = lb + (int64_t)i * a.sa;
        const int ix = (a.axis == 0) ? i : p0[0];
        const double x0 = (double)(ix - a.nl.shift0) * a.nl.dx0;
        double om = 0, ec = 1, es = 0;
        if (a.nl.kind == K_BRAGG) bragg_coupling(a.nl, x0, om, ec, es);
        C u[MAXC];
        u[0] = v[m];
        if (live) nl_point<R, TC>(a.nl, u, l, x0, om, ec, es);
        v[m] = u[0];
      }
    } else {
      __syncthreads();
      #pragma unroll
      for (int m = 0; m < 32; m++) {
        const int i = j + 16 * m;
        my[ex_at(i >> 4, i & 15)] = v[m];
      }
      __syncthreads();
      constexpr int PPT = 32 / TC;
      const bool bragg = (a.nl.kind == K_BRAGG);
      #pragma unroll 1  // as the 256-point passes: the rolled loop measured faster
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
      for (int m = 0; m < 32; m++) {
        const int i = j + 16 * m;
        v[m] = my[ex_at(i >> 4, i & 15)];
      }
    }
    p5_transform<R, -1>(v, my, twS, j);
  }

  if (live) {
    C *dst = f + lb + (int64_t)j * a.sa;
    #pragma unroll
    for (int m = 0; m < 32; m++) dst[m * step] = v[m];
  }
}

}  // namespace atus

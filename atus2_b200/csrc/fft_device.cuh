// fft_device.cuh -- shared-memory Stockham FFT building blocks for sm_100a.
//
// A CTA holds a tile of B pencils of length N (power of two, 2..8192) in shared
// memory, padded by one element every 16 so that the strided butterfly stores
// of a radix-16 pass spread over all banks.  A transform is a sequence of
// Stockham (self-sorting) passes of radix 16/8/4/2: every thread loads its
// butterflies' R inputs into registers, applies the twiddles and an R-point
// DFT, the CTA synchronises, and the thread stores the R outputs in their
// sorted positions.  Input and output are in natural order, so the passes can
// be fused with point-wise operators on either side.
//
// Direction: dir = -1 computes sum_j x_j exp(-2 pi i jk/N) (FFTW_FORWARD),
// dir = +1 the unnormalised inverse (FFTW_BACKWARD), the transform the
// reference calls through fftw_execute (source/libs/lib_myutils/cft_*d.cpp).
#pragma once
#include <cuda_runtime.h>

namespace atus {

template <typename R> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };
template <typename R> using cplx = typename cplx_t<R>::type;

template <typename R> __device__ __forceinline__ cplx<R> mk(R x, R y) { cplx<R> c; c.x = x; c.y = y; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  C r;
  r.x = a.x * b.x + a.y * b.y;
  r.y = a.y * b.x - a.x * b.y;
  return r;
}
// a * (dir * i)
template <int DIR, typename C> __device__ __forceinline__ C mul_i(C a) {
  C r;
  if (DIR < 0) { r.x = a.y; r.y = -a.x; }
  else { r.x = -a.y; r.y = a.x; }
  return r;
}

// Shared-memory index of element i of pencil b: one pad element per 16 inside
// a pencil (radix-16 stores), and an odd pencil pitch NP so that the same
// element of consecutive pencils falls into different banks (tile loads that
// walk across pencils, and the cluster transposes).
template <int N> struct Pad {
  static constexpr int NP = ((N >= 16) ? (N + N / 16) : N) | 1;
  static __device__ __forceinline__ int idx(int b, int i) { return b * NP + ((N >= 16) ? (i + (i >> 4)) : i); }
  static constexpr int words(int B) { return B * NP; }
};

// ---------------------------------------------------------------- small DFTs
template <int DIR, typename C> __device__ __forceinline__ void dft2(C *v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int DIR, typename C> __device__ __forceinline__ void dft4(C &a0, C &a1, C &a2, C &a3) {
  C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_i<DIR>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}
template <int DIR, typename C> __device__ __forceinline__ void dft4(C *v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }

// x * k for a compile-time constant k given in FP64.  In FP32 the constant
// is split k = hi + lo and the product formed as fma(x, hi, x lo): the
// rounding error of a float constant would otherwise be the same in every
// transform and bias the norm the same way each step.
__device__ __forceinline__ double kmul(double x, double k) { return x * k; }
__device__ __forceinline__ float kmul(float x, double k) {
  const float hi = (float)k;
  const float lo = (float)(k - (double)hi);
  return fmaf(x, hi, x * lo);
}

// exp(DIR * 2 pi i * m / 8) * a for m = 1, 3 (m = 2 is mul_i).
constexpr double SQRT1_2 = 0.70710678118654752440;
template <int DIR, typename C> __device__ __forceinline__ C w8_1(C a) {
  C r;  // (1 + DIR i) / sqrt 2
  if (DIR < 0) { r.x = kmul(a.x + a.y, SQRT1_2); r.y = kmul(a.y - a.x, SQRT1_2); }
  else { r.x = kmul(a.x - a.y, SQRT1_2); r.y = kmul(a.x + a.y, SQRT1_2); }
  return r;
}
template <int DIR, typename C> __device__ __forceinline__ C w8_3(C a) {
  C r;  // (-1 + DIR i) / sqrt 2
  if (DIR < 0) { r.x = kmul(a.y - a.x, SQRT1_2); r.y = -kmul(a.x + a.y, SQRT1_2); }
  else { r.x = -kmul(a.x + a.y, SQRT1_2); r.y = kmul(a.x - a.y, SQRT1_2); }
  return r;
}

template <int DIR, typename C> __device__ __forceinline__ void dft8(C *v) {
  // X[k] = E[k] + W8^k O[k], E/O = 4-point DFTs of even/odd samples
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<DIR>(e0, e1, e2, e3);
  dft4<DIR>(o0, o1, o2, o3);
  o1 = w8_1<DIR>(o1);
  o2 = mul_i<DIR>(o2);
  o3 = w8_3<DIR>(o3);
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// 16-point DFT as 4 x 4: X[m + 4p] = sum_q W4^{qp} W16^{qm} sum_s v[q+4s] W4^{sm}
template <int DIR, typename C> __device__ __forceinline__ void dft16(C *v) {
  using R = decltype(v[0].x);
  constexpr double c1 = 0.92387953251128675613;  // cos(pi/8)
  constexpr double s1 = 0.38268343236508977173;  // sin(pi/8)
  constexpr double ds1 = DIR * s1, dc1 = DIR * c1;
  #pragma unroll
  for (int q = 0; q < 4; q++) dft4<DIR>(v[q], v[q + 4], v[q + 8], v[q + 12]);
  // twiddles W16^{q m}: element (q, m) lives in v[q + 4m]
  {  // q = 1: m = 1, 2, 3 -> W16^1, W16^2, W16^3
    C a = v[5];
    v[5] = mk<R>(kmul(a.x, c1) - kmul(a.y, ds1), kmul(a.y, c1) + kmul(a.x, ds1));
    v[9] = w8_1<DIR>(v[9]);
    a = v[13];
    v[13] = mk<R>(kmul(a.x, s1) - kmul(a.y, dc1), kmul(a.y, s1) + kmul(a.x, dc1));
  }
  {  // q = 2: W16^2, W16^4, W16^6
    v[6] = w8_1<DIR>(v[6]);
    v[10] = mul_i<DIR>(v[10]);
    v[14] = w8_3<DIR>(v[14]);
  }
  {  // q = 3: W16^3, W16^6, W16^9
    C a = v[7];
    v[7] = mk<R>(kmul(a.x, s1) - kmul(a.y, dc1), kmul(a.y, s1) + kmul(a.x, dc1));
    v[11] = w8_3<DIR>(v[11]);
    a = v[15];  // W16^9 = exp(DIR i 9 pi/8) = -cos(pi/8) - DIR i sin(pi/8)
    v[15] = mk<R>(kmul(a.y, ds1) - kmul(a.x, c1), -kmul(a.y, c1) - kmul(a.x, ds1));
  }
  C o[16];
  #pragma unroll
  for (int m = 0; m < 4; m++) {
    C a0 = v[4 * m], a1 = v[4 * m + 1], a2 = v[4 * m + 2], a3 = v[4 * m + 3];
    dft4<DIR>(a0, a1, a2, a3);
    o[m] = a0; o[m + 4] = a1; o[m + 8] = a2; o[m + 12] = a3;
  }
  #pragma unroll
  for (int k = 0; k < 16; k++) v[k] = o[k];
}

template <int R_, int DIR, typename C> __device__ __forceinline__ void dftR(C *v) {
  if constexpr (R_ == 2) dft2<DIR>(v);
  else if constexpr (R_ == 4) dft4<DIR>(v);
  else if constexpr (R_ == 8) dft8<DIR>(v);
  else dft16<DIR>(v);
}

// Radix of pass p for length N: radix-16 passes first, then one 8, 4 or 2.
__host__ __device__ constexpr int lg2c(int n) { return n <= 1 ? 0 : 1 + lg2c(n / 2); }
__host__ __device__ constexpr int n_passes(int N) { return (lg2c(N) + 3) / 4; }
__host__ __device__ constexpr int pass_radix(int N, int p) {
  return (p < lg2c(N) / 4) ? 16 : (1 << (lg2c(N) - 4 * (lg2c(N) / 4)));
}
__host__ __device__ constexpr int pass_ns(int N, int p) {  // product of radices before pass p
  return p == 0 ? 1 : pass_ns(N, p - 1) * pass_radix(N, p - 1);
}

// Twiddle tables: exp(-2 pi i m / TWN) as double2 for FP64 transforms, and as
// float4 (hi.x, hi.y, lo.x, lo.y) with hi + lo = the FP64 value for FP32
// transforms, multiplied in compensated form (see kmul).
template <typename R> struct TwTab;
template <> struct TwTab<double> { using type = double2; };
template <> struct TwTab<float> { using type = float4; };

template <int DIR> __device__ __forceinline__ double2 twmul(double2 v, double2 w) {
  return (DIR < 0) ? cmul(v, w) : cmulc(v, w);
}
template <int DIR> __device__ __forceinline__ float2 twmul(float2 v, float4 w) {
  const float wy = DIR < 0 ? w.y : -w.y, ly = DIR < 0 ? w.w : -w.w;
  float2 r;
  r.x = fmaf(v.x, w.x, fmaf(-v.y, wy, v.x * w.z - v.y * ly));
  r.y = fmaf(v.x, wy, fmaf(v.y, w.x, v.x * ly + v.y * w.z));
  return r;
}

// One Stockham pass over B pencils held in shared memory.  tw is the global
// twiddle table exp(-2 pi i m / TWN), m in [0, TWN).
template <typename R, int N, int B, int NT, int RAD, int NS, int DIR, int TWN>
__device__ __forceinline__ void stockham_pass(cplx<R> *s, const typename TwTab<R>::type *__restrict__ tw) {
  using C = cplx<R>;
  using P = Pad<N>;
  constexpr int NB = B * N / RAD;                 // butterflies in the tile
  constexpr int PER = (NB + NT - 1) / NT;         // butterflies per thread
  constexpr int TWS = TWN / (NS * RAD);           // twiddle stride
  C v[PER][RAD];
  #pragma unroll
  for (int u = 0; u < PER; u++) {
    const int bf = threadIdx.x + u * NT;
    if (NB % NT == 0 || bf < NB) {
      const int b = bf / (N / RAD), j = bf % (N / RAD);
      const int k = j & (NS - 1);
      #pragma unroll
      for (int r = 0; r < RAD; r++) v[u][r] = s[P::idx(b, j + r * (N / RAD))];
      if (NS > 1) {
        #pragma unroll
        for (int r = 1; r < RAD; r++) {
          v[u][r] = twmul<DIR>(v[u][r], __ldg(&tw[(r * k) * TWS]));
        }
      }
      dftR<RAD, DIR>(v[u]);
    }
  }
  __syncthreads();
  #pragma unroll
  for (int u = 0; u < PER; u++) {
    const int bf = threadIdx.x + u * NT;
    if (NB % NT == 0 || bf < NB) {
      const int b = bf / (N / RAD), j = bf % (N / RAD);
      const int k = j & (NS - 1);
      const int o = (j / NS) * NS * RAD + k;
      #pragma unroll
      for (int r = 0; r < RAD; r++) s[P::idx(b, o + r * NS)] = v[u][r];
    }
  }
  __syncthreads();
}

template <typename R, int N, int B, int NT, int DIR, int TWN, int P>
__device__ __forceinline__ void fft_passes(cplx<R> *s, const typename TwTab<R>::type *__restrict__ tw) {
  if constexpr (P < n_passes(N)) {
    stockham_pass<R, N, B, NT, pass_radix(N, P), pass_ns(N, P), DIR, TWN>(s, tw);
    fft_passes<R, N, B, NT, DIR, TWN, P + 1>(s, tw);
  }
}

// In-place transform of the B pencils in shared memory (natural order in and
// out).  Caller synchronises before (data written) -- the first pass reads.
template <typename R, int N, int B, int NT, int DIR, int TWN>
__device__ __forceinline__ void fft_tile(cplx<R> *s, const typename TwTab<R>::type *__restrict__ tw) {
  if constexpr (N > 1) fft_passes<R, N, B, NT, DIR, TWN, 0>(s, tw);
}

}  // namespace atus

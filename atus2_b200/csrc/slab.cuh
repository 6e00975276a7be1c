// slab.cuh -- the (y,z)-slab pass of 3D grids on a thread-block cluster.
//
// One cluster of CS CTAs owns one x-slab (all y, z of one x index, every
// component).  A 256^2 slab of two complex128 components is 2 MB, more than
// one SM holds, so the slab is spread over the cluster's shared memory:
//
//   tile A (per CTA): ZB = NZ/CS z-columns, every y   -> y-transforms
//   tile B (per CTA): YB = NY/CS y-rows,    every z   -> z-transforms and the
//                                                       point-wise potential step
//
// and the CTAs swap between the two layouts through distributed shared memory
// (each thread pulls its elements from the owning CTA into registers, the
// cluster synchronises, then the elements are stored in the new layout).  A
// full pass  IFFT_y -> IFFT_z -> potential -> FFT_z -> FFT_y  therefore reads
// and writes each field once in HBM, instead of three times for three
// separate axis passes.  Variants without some of the stages handle the first
// (forward transforms only) and last (inverse only) pass of a Strang block.
// No TMA multicast is used anywhere.
#pragma once
#include <cooperative_groups.h>

#include "kernels.cuh"

namespace atus {

namespace cg = cooperative_groups;

struct SlabArgs {
  void *psi[MAXC];
  int nc;           // components in use (<= TC)
  int load_rows;    // 1: load tile B directly (no y work before the z stages)
  int inv_y, inv_z, do_nl, fwd_z, fwd_y;
  int store_rows;   // 1: store tile B directly (no y work after the z stages)
  const void *tw;
  Geo g;
  NLArgs nl;
};

template <typename R, int NY, int NZ, int TC, int CS>
struct SlabCfg {
  static constexpr int NT = 512;
  static constexpr int ZB = NZ / CS, YB = NY / CS;
  static constexpr int NPY = Pad<NY>::NP, NPZ = Pad<NZ>::NP;
  static constexpr int ELEMS = TC * NY * NZ / CS;  // complex values per CTA
  static constexpr int PER = (ELEMS + NT - 1) / NT;
  static constexpr size_t smemA = sizeof(cplx<R>) * TC * ZB * NPY;
  static constexpr size_t smemB = sizeof(cplx<R>) * TC * YB * NPZ;
  static constexpr size_t smem = smemA > smemB ? smemA : smemB;
};

template <typename R, int NY, int NZ, int TC, int CS>
__global__ void __launch_bounds__(512) slab_kernel(SlabArgs a) {
  using C = cplx<R>;
  using Cfg = SlabCfg<R, NY, NZ, TC, CS>;
  constexpr int NT = Cfg::NT, ZB = Cfg::ZB, YB = Cfg::YB, NPY = Cfg::NPY, NPZ = Cfg::NPZ;
  constexpr int PER = Cfg::PER, ELEMS = Cfg::ELEMS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *s = reinterpret_cast<C *>(smem_raw);
  __shared__ double s_coup[3];

  cg::cluster_group cluster = cg::this_cluster();
  const int r = (int)cluster.block_rank();
  const int64_t x = blockIdx.x / CS;
  const int64_t base = x * (int64_t)NY * NZ;
  const typename TwTab<R>::type *tw = (const typename TwTab<R>::type *)a.tw;
  C *fld[TC];
  #pragma unroll
  for (int c = 0; c < TC; c++) fld[c] = (C *)a.psi[c];

  // ---------------------------------------------------------------- load
  // every load of a thread is issued before its first shared-memory store
  constexpr int LPC = ELEMS / TC / NT;  // loads per thread and component
  static_assert((ELEMS / TC) % NT == 0, "slab tile must be a multiple of the CTA size");
  #pragma unroll
  for (int c = 0; c < TC; c++) {
    C val[LPC];
    #pragma unroll
    for (int k = 0; k < LPC; k++) {
      const int e = threadIdx.x + k * NT;
      val[k] = mk<R>(0, 0);
      if (c < a.nc) {
        if (a.load_rows) val[k] = fld[c][base + (int64_t)(r * YB + e / NZ) * NZ + e % NZ];
        else val[k] = fld[c][base + (int64_t)(e / ZB) * NZ + r * ZB + e % ZB];
      }
    }
    #pragma unroll
    for (int k = 0; k < LPC; k++) {
      const int e = threadIdx.x + k * NT;
      if (a.load_rows) s[(c * YB + e / NZ) * NPZ + Pad<NZ>::idx(0, e % NZ)] = val[k];
      else s[(c * ZB + e % ZB) * NPY + Pad<NY>::idx(0, e / ZB)] = val[k];
    }
  }
  __syncthreads();

  C reg[PER];
  if (!a.load_rows) {
    if (a.inv_y) fft_tile<R, NY, TC * ZB, NT, +1, TWN>(s, tw);
    // tile A -> tile B: element (c, yl, z) lives in CTA z/ZB at (c, z%ZB, r*YB+yl)
    cluster.sync();
    #pragma unroll
    for (int k = 0; k < PER; k++) {
      const int e = threadIdx.x + k * NT;
      if (ELEMS % NT == 0 || e < ELEMS) {
        const int yl = e % YB, z = (e / YB) % NZ, c = e / (YB * NZ);
        const C *rem = cluster.map_shared_rank(s, (unsigned)(z / ZB));
        reg[k] = rem[(c * ZB + (z % ZB)) * NPY + Pad<NY>::idx(0, r * YB + yl)];
      }
    }
    cluster.sync();
    #pragma unroll
    for (int k = 0; k < PER; k++) {
      const int e = threadIdx.x + k * NT;
      if (ELEMS % NT == 0 || e < ELEMS) {
        const int yl = e % YB, z = (e / YB) % NZ, c = e / (YB * NZ);
        s[(c * YB + yl) * NPZ + Pad<NZ>::idx(0, z)] = reg[k];
      }
    }
    __syncthreads();
  }

  // ---------------------------------------------------------------- z stages
  if (a.inv_z) fft_tile<R, NZ, TC * YB, NT, +1, TWN>(s, tw);
  if (a.do_nl) {
    const double x0 = (double)(x - a.nl.shift0) * a.nl.dx0;
    if (a.nl.kind == K_BRAGG) {
      if (threadIdx.x == 0) {
        double om, ec, es;
        bragg_coupling(a.nl, x0, om, ec, es);
        s_coup[0] = om; s_coup[1] = ec; s_coup[2] = es;
      }
      __syncthreads();
    }
    const double om = (a.nl.kind == K_BRAGG) ? s_coup[0] : 0.0;
    const double ec = (a.nl.kind == K_BRAGG) ? s_coup[1] : 1.0;
    const double es = (a.nl.kind == K_BRAGG) ? s_coup[2] : 0.0;
    #pragma unroll 4
    for (int e = threadIdx.x; e < YB * NZ; e += NT) {
      const int z = e % NZ, yl = e / NZ;
      const int64_t l = base + (int64_t)(r * YB + yl) * NZ + z;
      C v[MAXC];
      #pragma unroll
      for (int c = 0; c < TC; c++) v[c] = s[(c * YB + yl) * NPZ + Pad<NZ>::idx(0, z)];
      nl_point<R, TC>(a.nl, v, l, x0, om, ec, es);
      #pragma unroll
      for (int c = 0; c < TC; c++) s[(c * YB + yl) * NPZ + Pad<NZ>::idx(0, z)] = v[c];
    }
    __syncthreads();
  }
  if (a.fwd_z) fft_tile<R, NZ, TC * YB, NT, -1, TWN>(s, tw);

  // ---------------------------------------------------------------- store
  if (a.store_rows) {
    #pragma unroll
    for (int c = 0; c < TC; c++)
      if (c < a.nc)
        #pragma unroll
        for (int k = 0; k < LPC; k++) {
          const int e = threadIdx.x + k * NT;
          const int z = e % NZ, yl = e / NZ;
          fld[c][base + (int64_t)(r * YB + yl) * NZ + z] = s[(c * YB + yl) * NPZ + Pad<NZ>::idx(0, z)];
        }
    return;
  }
  // tile B -> tile A: element (c, zl, y) lives in CTA y/YB at (c, y%YB, r*ZB+zl)
  cluster.sync();
  #pragma unroll
  for (int k = 0; k < PER; k++) {
    const int e = threadIdx.x + k * NT;
    if (ELEMS % NT == 0 || e < ELEMS) {
      const int zl = e % ZB, y = (e / ZB) % NY, c = e / (ZB * NY);
      const C *rem = cluster.map_shared_rank(s, (unsigned)(y / YB));
      reg[k] = rem[(c * YB + (y % YB)) * NPZ + Pad<NZ>::idx(0, r * ZB + zl)];
    }
  }
  cluster.sync();
  #pragma unroll
  for (int k = 0; k < PER; k++) {
    const int e = threadIdx.x + k * NT;
    if (ELEMS % NT == 0 || e < ELEMS) {
      const int zl = e % ZB, y = (e / ZB) % NY, c = e / (ZB * NY);
      s[(c * ZB + zl) * NPY + Pad<NY>::idx(0, y)] = reg[k];
    }
  }
  __syncthreads();
  if (a.fwd_y) fft_tile<R, NY, TC * ZB, NT, -1, TWN>(s, tw);
  #pragma unroll
  for (int c = 0; c < TC; c++)
    if (c < a.nc)
      #pragma unroll
      for (int k = 0; k < LPC; k++) {
        const int e = threadIdx.x + k * NT;
        const int zl = e % ZB, y = e / ZB;
        fld[c][base + (int64_t)y * NZ + r * ZB + zl] = s[(c * ZB + zl) * NPY + Pad<NY>::idx(0, y)];
      }
}

}  // namespace atus

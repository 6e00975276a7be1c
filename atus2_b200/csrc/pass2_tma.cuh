// pass2_tma.cuh -- strided register-staged passes whose tiles arrive by TMA.
//
// The same work items as pass2_kernel (B adjacent pencils of 64..256 points
// of one component along a strided axis, one row of B values per point), but
// each tile is copied by one cp.async.bulk.tensor (a 3D box {B pencils, N
// points, 1}) into a shared-memory buffer -- 128-byte rows with 128-byte
// swizzle, longer rows plain -- complete on an mbarrier.  Once every thread
// has taken its 16 values from the buffer (conflict-free: a quarter warp
// reads consecutive pencils of one row, spread over the banks), one
// thread issues the copy of the CTA's next tile into it, so that copy flies
// while this tile is transformed and stored.  Waits on the mbarrier are
// bounded (PassArgs::wait_limit rounds of try_wait): on time-out every thread
// leaves the loop and the error word is set (read by the host after the
// block).  A copy that never lands thus ends the pass with an error status
// instead of a hang; PassArgs::drop_copies (no copy issued, no arrival on
// the barrier) makes every wait run out with nothing in flight, for tests of
// that path.
#pragma once
#include <cuda.h>

#include "pass2.cuh"

namespace atus {

// One tensor map per component (cuTensorMapEncodeTiled on the host).
struct alignas(64) TmaMaps {
  CUtensorMap m[MAXC];
};

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned mbar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned mbar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}
// 3D tile load, no multicast: box at coordinates {c0, c1, c2} of `map` into
// shared memory at dst, completing `bytes` on mbar.
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            unsigned mbar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(mbar)
      : "memory");
}

template <typename R, int N>
struct P2TmaCfg {
  using Cfg = P2Cfg<R, N, 1>;
  static constexpr int B = Cfg::B;
  static constexpr int VPC = (int)sizeof(cplx<R>) / 8;  // 8-byte units per value
  static constexpr int ROW = B * (int)sizeof(cplx<R>);  // bytes per point of the tile
  static constexpr unsigned TILE_BYTES = (unsigned)N * ROW;
  static constexpr bool SWZ = (ROW == 128);               // 128-byte swizzle (else none)
  static_assert(ROW >= 128 && VPC * B <= 256, "rows of 128 bytes or more, at most 256 units a box row");
  // tile (1024-byte aligned inside the allocation) + exchange rows + twiddles
  static constexpr size_t smem = 1024 + TILE_BYTES + Cfg::smem;
};

template <typename R, int N, int MODE>
__global__ void __launch_bounds__(Tile2<R>::NT, 3) pass2_tma_kernel(PassArgs a, const __grid_constant__ TmaMaps maps) {
  using T = P2TmaCfg<R, N>;
  constexpr int B = T::B;
  extern __shared__ __align__(16) unsigned char smem_all[];
  const unsigned base = smem_u32(smem_all);
  unsigned char *const tile = smem_all + ((1024u - (base & 1023u)) & 1023u);
  unsigned char *const rest = tile + T::TILE_BYTES;
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ double s_om[B], s_ec[B], s_es[B];
  const unsigned mb = smem_u32(&mbar);
  const int tid = threadIdx.x;
  p2_setup<R, N, 1, M2_FWD>(a, rest);  // twiddle rows only (kinetic factors from global)
  if (tid == 0) {
    mbar_init(mb, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const int64_t W = a.ntiles * a.ncomp_grid;
  auto issue = [&](int64_t w) {
    const int comp = (int)(w / a.ntiles);
    const int64_t t = w % a.ntiles;
    const int o = (int)(t / a.inner_tiles);
    const int r0 = (int)((t % a.inner_tiles) * B);
    if (a.drop_copies) return;  // the barrier phase then never completes
    mbar_expect_tx(mb, T::TILE_BYTES);
    tma_load_3d(smem_u32(tile), &maps.m[comp], T::VPC * r0, 0, o, mb);
  };
  int64_t w = blockIdx.x;
  if (tid == 0 && w < W) issue(w);
  unsigned parity = 0;
  for (; w < W; w += gridDim.x) {
    bool ok = false;
    for (long it = 0; it < a.wait_limit && !ok; it++) ok = mbar_try_wait(mb, parity);
    if (!__syncthreads_and(ok)) {
      if (tid == 0 && a.err) atomicOr(a.err, 1);
      break;
    }
    parity ^= 1;
    const int64_t wn = w + gridDim.x;
    auto refill = [&]() {
      __syncthreads();  // every thread has its values: the buffer is free
      if (tid == 0 && wn < W) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(wn);
      }
    };
    p2_item<R, N, 1, MODE, true, true>(a, tile_geo<B, N>(a, w), rest, false, s_om, s_ec, s_es, nullptr, tile,
                                       refill);
  }
}

}  // namespace atus

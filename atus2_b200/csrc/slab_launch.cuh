// slab_launch.cuh -- launcher of the cluster slab pass (see slab.cuh).
#pragma once
#include "ctx.h"
#include "slab.cuh"

// Cluster size: enough CTAs that each holds at most 64 KB of the slab
// (128 KB for the two-component complex128 256^2 slab, where 16 is the
// largest cluster the hardware schedules).
template <typename R, int N, int TC>
struct SlabCS {
  static constexpr long bytes = (long)sizeof(cplx<R>) * TC * N * N;
  static constexpr int raw = (int)(bytes / 65536);
  static constexpr int value = raw < 2 ? 2 : (raw > 16 ? 16 : raw);
};

template <typename R, int N, int TC>
static inline int launch_slab_t(atus_ctx *ctx, SlabArgs &a) {
  constexpr int CS = SlabCS<R, N, TC>::value;
  using Cfg = SlabCfg<R, N, N, TC, CS>;
  auto kern = slab_kernel<R, N, N, TC, CS>;
  static int state = 0;  // 0 unknown, 1 usable, -1 not schedulable
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(ctx->n[0] * CS));
  cfg.blockDim = dim3(Cfg::NT);
  cfg.dynamicSmemBytes = Cfg::smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (state == 0) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem) != cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) !=
            cudaSuccess ||
        (CS > 8 && cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
      cudaGetLastError();
      state = -1;
    } else {
      int nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1) {
        cudaGetLastError();
        state = -1;
      } else {
        state = 1;
      }
    }
  }
  if (state < 0) return ATUS_E_UNSUPPORTED;
  a.tw = (sizeof(R) == 8) ? ctx->tw64 : ctx->tw;
  a.g = geo(ctx);
  CK(cudaLaunchKernelEx(&cfg, kern, a));
  LAUNCHED(ctx);
  return ATUS_OK;
}

template <typename R, int TC>
static inline int launch_slab_n(atus_ctx *ctx, SlabArgs &a) {
  if (ctx->dim != 3 || ctx->n[1] != ctx->n[2]) return ATUS_E_UNSUPPORTED;
  switch (ctx->n[1]) {
    case 32: return launch_slab_t<R, 32, TC>(ctx, a);
    case 64: return launch_slab_t<R, 64, TC>(ctx, a);
    case 128: return launch_slab_t<R, 128, TC>(ctx, a);
    case 256: return launch_slab_t<R, 256, TC>(ctx, a);
    default: return ATUS_E_UNSUPPORTED;
  }
}

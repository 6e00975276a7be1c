// launch.cuh -- launchers of the templated kernels.  Each instantiation file
// (inst_*.cu) includes this and exports one precision / component-count
// combination, so the kernels compile in parallel.
#pragma once
#include <cstring>

#include "ctx.h"
#include "cluster1d.cuh"
#include "pass2.cuh"
#include "pass2_tma.cuh"
#include "pass3.cuh"

template <typename R, int N, int TC>
static inline int launch_pass_t(atus_ctx *ctx, PassArgs &a, int axis) {
  using Cfg = PassCfg<R, N, TC>;
  constexpr size_t smem = Cfg::smem;
  if (smem + 3 * sizeof(double) * Cfg::B > 227 * 1024) return fail(ctx, ATUS_E_UNSUPPORTED, "pencil too long for this component count");
  static int resident = 0;  // CTAs of this instantiation per SM
  static int nsm = 0;
  if (!resident) {
    CK(cudaFuncSetAttribute(pass_kernel<R, N, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // all of the unified L1/shared storage as shared memory: the tiles are
    // the working set, global accesses are streaming
    CK(cudaFuncSetAttribute(pass_kernel<R, N, TC>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, pass_kernel<R, N, TC>, Cfg::NT, smem));
    if (resident < 1) return fail(ctx, ATUS_E_UNSUPPORTED, "pass kernel does not fit on an SM");
  }
  int64_t sa = 1;
  for (int b = axis + 1; b < 3; b++) sa *= ctx->n[b];
  a.sa = sa;
  int64_t ntiles;
  if (sa > 1) {
    a.inner_tiles = (sa + Cfg::B - 1) / Cfg::B;
    ntiles = (ctx->npts / (N * sa)) * a.inner_tiles;
    a.npencils = 0;
  } else {
    a.inner_tiles = 1;
    a.npencils = ctx->npts / N;
    ntiles = (a.npencils + Cfg::B - 1) / Cfg::B;
  }
  a.x_along = (axis == 0);
  a.axis = axis;
  a.g = geo(ctx);
  a.tw = (sizeof(R) == 8) ? ctx->tw64 : ctx->tw;
  for (int ax = 0; ax < 3; ax++) {
    a.dk[ax] = ctx->dk[ax];
    a.n[ax] = (int)ctx->n[ax];
  }
  a.ntiles = ntiles;
  a.ncomp_grid = ctx->ncomp;
  // persistent grid: every resident CTA walks work items with stride gridDim
  const int64_t work = a.per_comp ? ntiles * ctx->ncomp : ntiles;
  const int64_t slots = (int64_t)nsm * resident;
  const unsigned grid = (unsigned)(work < slots ? work : slots);
  pass_kernel<R, N, TC><<<grid, Cfg::NT, smem, ctx->stream>>>(a);
  LAUNCHED(ctx);
  return ATUS_OK;
}

template <typename R, int TC>
static inline int launch_pass_n(atus_ctx *ctx, PassArgs &a, int axis) {
  switch (ctx->n[axis]) {
    case 2: return launch_pass_t<R, 2, TC>(ctx, a, axis);
    case 4: return launch_pass_t<R, 4, TC>(ctx, a, axis);
    case 8: return launch_pass_t<R, 8, TC>(ctx, a, axis);
    case 16: return launch_pass_t<R, 16, TC>(ctx, a, axis);
    case 32: return launch_pass_t<R, 32, TC>(ctx, a, axis);
    case 64: return launch_pass_t<R, 64, TC>(ctx, a, axis);
    case 128: return launch_pass_t<R, 128, TC>(ctx, a, axis);
    case 256: return launch_pass_t<R, 256, TC>(ctx, a, axis);
    case 512: return launch_pass_t<R, 512, TC>(ctx, a, axis);
    case 1024: return launch_pass_t<R, 1024, TC>(ctx, a, axis);
    case 2048: return launch_pass_t<R, 2048, TC>(ctx, a, axis);
    case 4096: return launch_pass_t<R, 4096, TC>(ctx, a, axis);
    case 8192: return launch_pass_t<R, 8192, TC>(ctx, a, axis);
    default: return fail(ctx, ATUS_E_UNSUPPORTED, "axis length must be a power of two in [2, 8192]");
  }
}

template <typename R, int N, int TC>
static inline int launch_block1d_t(atus_ctx *ctx, Block1DArgs &a) {
  constexpr size_t smem = sizeof(cplx<R>) * TC * Pad<N>::NP;
  if (smem > 227 * 1024) return fail(ctx, ATUS_E_UNSUPPORTED, "1D grid too long for the resident kernel");
  static bool attr_set = false;
  if (!attr_set) {
    CK(cudaFuncSetAttribute(block1d_kernel<R, N, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_set = true;
  }
  block1d_kernel<R, N, TC><<<1, BLOCK1D_NT, smem, ctx->stream>>>(a);
  LAUNCHED(ctx);
  return ATUS_OK;
}

// A 1D block on one cluster of CTAs (cluster1d.cuh).
// ATUS_E_UNSUPPORTED (nothing launched) where the device cannot place such a
// cluster (then the caller takes the one-CTA kernel or the per-step passes).
template <typename R, int N, int TC>
static inline int launch_cluster1d_t(atus_ctx *ctx, Block1DArgs &a) {
  using Cfg = C1Cfg<R, N, TC>;
  static int placeable = -1;  // clusters of this kernel the device can hold at once
  if (placeable < 0) {
    CK(cudaFuncSetAttribute(cluster1d_kernel<R, N, TC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::smem));
    if (Cfg::C > 8) CK(cudaFuncSetAttribute(cluster1d_kernel<R, N, TC>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(Cfg::C);
    cfg.blockDim = dim3(Cfg::NT);
    cfg.dynamicSmemBytes = Cfg::smem;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = Cfg::C;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int n = 0;
    placeable = (cudaOccupancyMaxActiveClusters(&n, cluster1d_kernel<R, N, TC>, &cfg) == cudaSuccess) ? n : 0;
    cudaGetLastError();  // a refused query leaves no sticky error
  }
  if (placeable < 1) return ATUS_E_UNSUPPORTED;
  cluster1d_kernel<R, N, TC><<<Cfg::C, Cfg::NT, Cfg::smem, ctx->stream>>>(a);
  LAUNCHED(ctx);
  return ATUS_OK;
}

template <typename R, int TC>
static inline int launch_block1d_n(atus_ctx *ctx, Block1DArgs &a) {
  if (ctx->use_cluster1d) {
    int r = ATUS_E_UNSUPPORTED;
    switch (ctx->n[0]) {
      case 2048: r = launch_cluster1d_t<R, 2048, TC>(ctx, a); break;
      case 4096: r = launch_cluster1d_t<R, 4096, TC>(ctx, a); break;
      case 8192: r = launch_cluster1d_t<R, 8192, TC>(ctx, a); break;
      default: break;
    }
    if (r != ATUS_E_UNSUPPORTED) return r;
  }
  switch (ctx->n[0]) {
    case 2: return launch_block1d_t<R, 2, TC>(ctx, a);
    case 4: return launch_block1d_t<R, 4, TC>(ctx, a);
    case 8: return launch_block1d_t<R, 8, TC>(ctx, a);
    case 16: return launch_block1d_t<R, 16, TC>(ctx, a);
    case 32: return launch_block1d_t<R, 32, TC>(ctx, a);
    case 64: return launch_block1d_t<R, 64, TC>(ctx, a);
    case 128: return launch_block1d_t<R, 128, TC>(ctx, a);
    case 256: return launch_block1d_t<R, 256, TC>(ctx, a);
    case 512: return launch_block1d_t<R, 512, TC>(ctx, a);
    case 1024: return launch_block1d_t<R, 1024, TC>(ctx, a);
    case 2048: return launch_block1d_t<R, 2048, TC>(ctx, a);
    case 4096: return launch_block1d_t<R, 4096, TC>(ctx, a);
    case 8192: return launch_block1d_t<R, 8192, TC>(ctx, a);
    default: return fail(ctx, ATUS_E_UNSUPPORTED, "axis length must be a power of two in [2, 8192]");
  }
}


// ------------------------------------------------------------ register-staged passes
// Launch of pass2_kernel (pencils of 32..256 points); ATUS_E_UNSUPPORTED,
// without an error message, for lengths it has no instantiation for.
// cuTensorMapEncodeTiled from the driver (no link against libcuda).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static inline EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// Strided pass with TMA tile copies (pass2_tma.cuh); the tile and
// launch geometry of launch_pass2_t.  ATUS_E_UNSUPPORTED (nothing launched)
// where a tensor map cannot describe the pass.
template <typename R, int N, int MODE>
static inline int launch_pass2_tma_t(atus_ctx *ctx, PassArgs &a, int axis) {
  using T = P2TmaCfg<R, N>;
  constexpr size_t smem = T::smem;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return ATUS_E_UNSUPPORTED;
  int64_t sa = 1;
  for (int b = axis + 1; b < 3; b++) sa *= ctx->n[b];
  const int64_t outer = ctx->npts / (N * sa);
  // whole tiles only (the box never reaches past the row), coordinates in int32
  if (sa < T::B || sa % T::B != 0 || T::VPC * sa > (int64_t(1) << 31) || outer > (int64_t(1) << 31))
    return ATUS_E_UNSUPPORTED;
  static int resident = 0;
  static int nsm = 0;
  if (!resident) {
    CK(cudaFuncSetAttribute(pass2_tma_kernel<R, N, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(cudaFuncSetAttribute(pass2_tma_kernel<R, N, MODE>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, pass2_tma_kernel<R, N, MODE>, T::Cfg::NT, smem));
    if (resident < 1) return fail(ctx, ATUS_E_UNSUPPORTED, "TMA pass kernel does not fit on an SM");
  }
  const int nf = a.per_comp ? ctx->ncomp : 1;
  TmaMaps maps;
  memset(&maps, 0, sizeof(maps));
  for (int c = 0; c < nf; c++) {
    // 8-byte units: {VPC sa, N, outer}, box {VPC B, N, 1}, 128-byte swizzle for 128-byte rows
    const cuuint64_t dims[3] = {(cuuint64_t)(T::VPC * sa), (cuuint64_t)N, (cuuint64_t)outer};
    const cuuint64_t strides[2] = {(cuuint64_t)(T::VPC * sa * 8), (cuuint64_t)(T::VPC * sa * 8 * N)};
    const cuuint32_t box[3] = {(cuuint32_t)(T::VPC * T::B), (cuuint32_t)N, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    if (enc(&maps.m[c], CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, a.psi[c], dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, T::SWZ ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return ATUS_E_UNSUPPORTED;
  }
  a.sa = sa;
  a.inner_tiles = (sa + T::B - 1) / T::B;
  const int64_t ntiles = outer * a.inner_tiles;
  a.npencils = 0;
  a.x_along = (axis == 0);
  a.axis = axis;
  a.g = geo(ctx);
  a.tw = (sizeof(R) == 8) ? ctx->tw64 : ctx->tw;
  for (int ax = 0; ax < 3; ax++) {
    a.dk[ax] = ctx->dk[ax];
    a.n[ax] = (int)ctx->n[ax];
  }
  a.ntiles = ntiles;
  a.ncomp_grid = ctx->ncomp;
  a.err = ctx->err_dev;
  a.wait_limit = ctx->wait_limit;
  a.drop_copies = ctx->drop_copies;
  const int64_t work = ntiles * ctx->ncomp;
  const int64_t slots = (int64_t)nsm * resident;
  const unsigned grid = (unsigned)(work < slots ? work : slots);
  pass2_tma_kernel<R, N, MODE><<<grid, T::Cfg::NT, smem, ctx->stream>>>(a, maps);
  LAUNCHED(ctx);
  ctx->err_armed = true;
  return ATUS_OK;
}

template <typename R, int N, int TC, int MODE, bool STRIDED>
static inline int launch_pass2_t(atus_ctx *ctx, PassArgs &a, int axis) {
  // 256-point pencils only: on 128-point pencils (the 128^3 Sobolev
  // iteration) the TMA-fed passes measured no faster (0.253 vs 0.252 ms per
  // iteration)
  if constexpr (STRIDED && N == 256 && TC == 1 && (MODE == M2_FWD || MODE == M2_INV || MODE == M2_KIN)) {
    if (ctx->use_tma && a.per_comp && ctx->err_dev && ctx->npts / ctx->n[axis] >= 2) {
      const int r = launch_pass2_tma_t<R, N, MODE>(ctx, a, axis);
      if (r != ATUS_E_UNSUPPORTED) return r;
    }
  }
  using Cfg = P2Cfg<R, N, TC>;
  constexpr size_t smem = ((MODE == M2_KIN || MODE == M2_KIN_RABI) && Cfg::kin_smem) ? Cfg::smem_kin : Cfg::smem;
  static int resident = 0;
  static int nsm = 0;
  if (!resident) {
    CK(cudaFuncSetAttribute(pass2_kernel<R, N, TC, MODE, STRIDED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem));
    CK(cudaFuncSetAttribute(pass2_kernel<R, N, TC, MODE, STRIDED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, pass2_kernel<R, N, TC, MODE, STRIDED>, Cfg::NT, smem));
    if (resident < 1) return fail(ctx, ATUS_E_UNSUPPORTED, "pass kernel does not fit on an SM");
  }
  int64_t sa = 1;
  for (int b = axis + 1; b < 3; b++) sa *= ctx->n[b];
  if ((sa > 1) != STRIDED) return ATUS_E_UNSUPPORTED;
  a.sa = sa;
  int64_t ntiles;
  if (sa > 1) {
    a.inner_tiles = (sa + Cfg::B - 1) / Cfg::B;
    ntiles = (ctx->npts / (N * sa)) * a.inner_tiles;
    a.npencils = 0;
  } else {
    a.inner_tiles = 1;
    a.npencils = ctx->npts / N;
    ntiles = (a.npencils + Cfg::B - 1) / Cfg::B;
  }
  a.x_along = (axis == 0);
  a.axis = axis;
  a.g = geo(ctx);
  a.tw = (sizeof(R) == 8) ? ctx->tw64 : ctx->tw;
  for (int ax = 0; ax < 3; ax++) {
    a.dk[ax] = ctx->dk[ax];
    a.n[ax] = (int)ctx->n[ax];
  }
  a.ntiles = ntiles;
  a.ncomp_grid = ctx->ncomp;
  const int64_t work = a.per_comp ? ntiles * ctx->ncomp : ntiles;
  const int64_t slots = (int64_t)nsm * resident;
  unsigned grid = (unsigned)(work < slots ? work : slots);
  if (MODE == M2_KIN_RABI && grid > RED_BLOCKS) grid = RED_BLOCKS;  // one partial row per CTA
  pass2_kernel<R, N, TC, MODE, STRIDED><<<grid, Cfg::NT, smem, ctx->stream>>>(a);
  LAUNCHED(ctx);
  return ATUS_OK;
}

// Launch of pass3_kernel (pencils of 512..2048 points); as launch_pass2_t.
template <typename R, int N, int TC, int MODE, bool STRIDED>
static inline int launch_pass3_t(atus_ctx *ctx, PassArgs &a, int axis) {
  using Cfg = P3Cfg<R, N, TC, STRIDED>;
  constexpr size_t smem = Cfg::smem;
  static int resident = 0;
  static int nsm = 0;
  if (!resident) {
    CK(cudaFuncSetAttribute(pass3_kernel<R, N, TC, MODE, STRIDED>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)smem));
    CK(cudaFuncSetAttribute(pass3_kernel<R, N, TC, MODE, STRIDED>, cudaFuncAttributePreferredSharedMemoryCarveout,
                            cudaSharedmemCarveoutMaxShared));
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, pass3_kernel<R, N, TC, MODE, STRIDED>, Cfg::NT, smem));
    if (resident < 1) return fail(ctx, ATUS_E_UNSUPPORTED, "pass kernel does not fit on an SM");
  }
  int64_t sa = 1;
  for (int b = axis + 1; b < 3; b++) sa *= ctx->n[b];
  if ((sa > 1) != STRIDED) return ATUS_E_UNSUPPORTED;
  a.sa = sa;
  int64_t ntiles;
  if (sa > 1) {
    a.inner_tiles = (sa + Cfg::B - 1) / Cfg::B;
    ntiles = (ctx->npts / (N * sa)) * a.inner_tiles;
    a.npencils = 0;
  } else {
    a.inner_tiles = 1;
    a.npencils = ctx->npts / N;
    ntiles = (a.npencils + Cfg::B - 1) / Cfg::B;
  }
  a.x_along = (axis == 0);
  a.axis = axis;
  a.g = geo(ctx);
  a.tw = (sizeof(R) == 8) ? ctx->tw64 : ctx->tw;
  for (int ax = 0; ax < 3; ax++) {
    a.dk[ax] = ctx->dk[ax];
    a.n[ax] = (int)ctx->n[ax];
  }
  a.ntiles = ntiles;
  a.ncomp_grid = ctx->ncomp;
  const int64_t work = a.per_comp ? ntiles * ctx->ncomp : ntiles;
  const int64_t slots = (int64_t)nsm * resident;
  const unsigned grid = (unsigned)(work < slots ? work : slots);
  pass3_kernel<R, N, TC, MODE, STRIDED><<<grid, Cfg::NT, smem, ctx->stream>>>(a);
  LAUNCHED(ctx);
  return ATUS_OK;
}

template <typename R, int TC, int MODE, bool STRIDED>
static inline int launch_pass2_n(atus_ctx *ctx, PassArgs &a, int axis) {
  switch (ctx->n[axis]) {
    case 32: return launch_pass2_t<R, 32, TC, MODE, STRIDED>(ctx, a, axis);
    case 64: return launch_pass2_t<R, 64, TC, MODE, STRIDED>(ctx, a, axis);
    case 128: return launch_pass2_t<R, 128, TC, MODE, STRIDED>(ctx, a, axis);
    case 256: return launch_pass2_t<R, 256, TC, MODE, STRIDED>(ctx, a, axis);
    default: break;
  }
  if constexpr (MODE != M2_KIN_RABI) {
    switch (ctx->n[axis]) {
      case 512: return launch_pass3_t<R, 512, TC, MODE, STRIDED>(ctx, a, axis);
      case 1024: return launch_pass3_t<R, 1024, TC, MODE, STRIDED>(ctx, a, axis);
      case 2048: return launch_pass3_t<R, 2048, TC, MODE, STRIDED>(ctx, a, axis);
      default: break;
    }
  }
  return ATUS_E_UNSUPPORTED;
}


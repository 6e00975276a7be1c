// noalloc.cu -- particle number of a device field without any allocation.
//
// atus_particle_number() reduces through the partial-sum buffer that
// atus_create() allocates with cudaMalloc.  Callers that cannot allocate
// device memory -- a host framework whose caching allocator or fixed pool owns
// the device memory, or a time step that cannot take the device-wide
// synchronisation of cudaFree -- use atus_particle_number_noalloc(): same sum,
// field by device pointer, no context, and its partial sums in the fixed
// device array below.  Nothing here calls cudaMalloc, cudaFree or any other
// allocating routine.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/atus_gpu.h"

namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_PER_THREAD = 128;
constexpr long long NA_CHUNK = (long long)NA_THREADS * NA_PER_THREAD;  // points per partial sum
constexpr int NA_MAX_CHUNKS = 4096;                                     // 32 KB of partial sums
static_assert(NA_CHUNK * NA_MAX_CHUNKS == ATUS_NOALLOC_MAX_POINTS, "limit and array size disagree");

// One partial sum per chunk of NA_CHUNK points, shared by every call on a
// device.  No entry has to start at zero: each entry a call reads is written
// by the first kernel of the same call.  Calls that overlap on the GPU race
// on these entries.
static __device__ __align__(256) double na_partials[NA_MAX_CHUNKS];

// Chunk b: fixed per-thread order, fixed tree -- the sum does not depend on
// the launch.
template <typename C>
__global__ void __launch_bounds__(NA_THREADS) na_chunk_kernel(const C *__restrict__ psi, long long npts,
                                                              double *__restrict__ partials) {
  const long long base = (long long)blockIdx.x * NA_CHUNK;
  double s = 0.0;
  #pragma unroll 8
  for (int k = 0; k < NA_PER_THREAD; k++) {
    const long long l = base + (long long)k * NA_THREADS + threadIdx.x;
    if (l < npts) {
      const C v = psi[l];
      s += (double)v.x * (double)v.x + (double)v.y * (double)v.y;
    }
  }
  __shared__ double sh[NA_THREADS];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = NA_THREADS / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sh[0];
}

// One warp: lane i adds chunks i, i + 32, ... in order, lane 0 adds the 32
// lane sums in order and scales by the volume element.
__global__ void na_final_kernel(const double *__restrict__ partials, int nchunks, double ar, double *out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int c = threadIdx.x; c < nchunks; c += 32) s += partials[c];
  sh[threadIdx.x] = s;
  __syncwarp();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < 32; i++) t += sh[i];
    *out = ar * t;
  }
}

// Device address of na_partials, looked up once per device with that device
// current (the first call on the device does it), together with the id of the
// CUDA context it belongs to.  Context ids are never reused within a process,
// so after cudaDeviceReset (a new primary context, the module loaded again at
// another address) the next call sees a different id and looks the address
// up again instead of launching with a stale one.
constexpr int NA_MAX_DEVICES = 64;
struct NaSlot {
  unsigned long long ctx_id;
  double *addr;
};
NaSlot na_slot[NA_MAX_DEVICES];
std::mutex na_mu;

// cuCtxGetCurrent and cuCtxGetId through the runtime's driver entry points
// (no link against the driver library); null where the driver lacks them.
using CtxGetCurrentFn = int (*)(void **);
using CtxGetIdFn = int (*)(void *, unsigned long long *);
template <typename F> F na_driver_fn(const char *name) {
  void *fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPointByVersion(name, &fn, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(fn);
}

// Id of the calling thread's current context; false when there is none yet
// (the runtime creates the primary context on its first real call) or the
// driver cannot tell.
bool na_current_ctx(unsigned long long *id) {
  static const CtxGetCurrentFn get_cur = na_driver_fn<CtxGetCurrentFn>("cuCtxGetCurrent");
  static const CtxGetIdFn get_id = na_driver_fn<CtxGetIdFn>("cuCtxGetId");
  void *ctx = nullptr;
  if (!get_cur || !get_id || get_cur(&ctx) != 0 || !ctx) return false;
  return get_id(ctx, id) == 0;
}

}  // namespace

extern "C" ATUS_API int atus_particle_number_noalloc(const void *psi_dev, int64_t npts, int precision, double ar,
                                                     double *out_dev, void *stream) {
  if (!out_dev || npts < 0 || (npts > 0 && !psi_dev)) return ATUS_E_ARG;
  if (precision != ATUS_PREC_FP64 && precision != ATUS_PREC_MIXED) return ATUS_E_ARG;
  if (npts > ATUS_NOALLOC_MAX_POINTS) return ATUS_E_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return ATUS_E_CUDA;
  double *partials = nullptr;
  {
    std::lock_guard<std::mutex> lock(na_mu);
    unsigned long long id = 0;
    const bool known = na_current_ctx(&id);
    NaSlot &slot = na_slot[dev];
    if (!slot.addr || !known || slot.ctx_id != id) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, na_partials) != cudaSuccess || !p) return ATUS_E_CUDA;
      // the lookup made the device's context current; without a context id
      // the address is not cached and every call looks it up
      slot.addr = na_current_ctx(&id) ? static_cast<double *>(p) : nullptr;
      slot.ctx_id = id;
      partials = static_cast<double *>(p);
    } else {
      partials = slot.addr;
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nchunks = (int)((npts + NA_CHUNK - 1) / NA_CHUNK);
  if (nchunks > 0) {
    if (precision == ATUS_PREC_FP64)
      na_chunk_kernel<double2><<<nchunks, NA_THREADS, 0, s>>>(static_cast<const double2 *>(psi_dev), npts, partials);
    else
      na_chunk_kernel<float2><<<nchunks, NA_THREADS, 0, s>>>(static_cast<const float2 *>(psi_dev), npts, partials);
    if (cudaGetLastError() != cudaSuccess) return ATUS_E_CUDA;
  }
  na_final_kernel<<<1, 32, 0, s>>>(partials, nchunks, ar, out_dev);
  if (cudaGetLastError() != cudaSuccess) return ATUS_E_CUDA;
  return ATUS_OK;
}

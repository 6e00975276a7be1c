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
// current (the first call on the device does it).
constexpr int NA_MAX_DEVICES = 64;
double *na_addr[NA_MAX_DEVICES];
std::mutex na_mu;

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
    if (!na_addr[dev]) {
      void *p = nullptr;
      if (cudaGetSymbolAddress(&p, na_partials) != cudaSuccess || !p) return ATUS_E_CUDA;
      na_addr[dev] = static_cast<double *>(p);
    }
    partials = na_addr[dev];
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

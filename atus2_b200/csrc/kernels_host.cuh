// kernels_host.cuh -- non-template kernels, compiled once (in capi.cu).
#pragma once
#include "kernels.cuh"

namespace atus {

__global__ void sob_assemble_kernel(SobArgs a) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < a.npts; l += (int64_t)gridDim.x * blockDim.x) {
    double nl = 0;
    #pragma unroll
    for (int j = 0; j < MAXC; j++) {
      if (j < a.ncomp) {
        const double2 p = a.psi[j][l];
        nl += a.gs[a.comp * MAXC + j] * (p.x * p.x + p.y * p.y);
      }
    }
    const double pot = a.V ? a.V[l] : 0.0;
    const double2 p = a.psi[a.comp][l], L = a.lap[l];
    a.grad[l] = make_double2(-L.x + (pot + nl) * p.x, -L.y + (pot + nl) * p.y);
  }
}

// y -= f * x
__global__ void axpy_kernel(double2 *y, const double2 *x, double f, int64_t n) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    double2 v = y[l];
    const double2 u = x[l];
    v.x -= f * u.x;
    v.y -= f * u.y;
    y[l] = v;
  }
}

__global__ void scale_kernel(double2 *y, double f, int64_t n) {
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    double2 v = y[l];
    v.x *= f;
    v.y *= f;
    y[l] = v;
  }
}

__global__ void reduce_final(const double *partial, int nblocks, int nq, double *out) {
  const int i = threadIdx.x;
  if (i < nq) {
    double s = 0;
    for (int b = 0; b < nblocks; b++) s += partial[b * RED_MAXQ + i];
    out[i] = s;
  }
}

}  // namespace atus

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
    const double2 p = a.psi[a.comp][l];
    if (a.copy) a.copy[l] = p;
    if (a.lap) {
      const double2 L = a.lap[l];
      a.grad[l] = make_double2(-L.x + (pot + nl) * p.x, -L.y + (pot + nl) * p.y);
    } else {  // the potential term alone (W psi)
      a.grad[l] = make_double2((pot + nl) * p.x, (pot + nl) * p.y);
    }
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

// ------------------------------------------------------------ Sobolev run on the device
// Scalars of the descent kept in device memory, so that a chunk of iterations
// runs (as a CUDA graph) without host round trips.  Per component: q = the two
// projections Re<psi, G>, Re<psi, psi_sob>; g2 = sum |G|^2; n = sum |psi|^2.
struct SobDev {
  double q[MAXC][3];    // Re<psi, G>, Re<psi, psi_sob>, <psi, psi> (one reduction)
  double g2[MAXC];
  double scale[MAXC];   // renormalisation factor of this iteration (1: none)
  double res;           // residual of the last active iteration
  double N[MAXC];       // particle numbers of the last active iteration
  double eps;
  int max_iter;
  int iters;            // iterations done
  int active;           // this iteration updates psi
  int stop;             // its residual is <= eps
  int done;             // no further iteration updates psi
};

// G -= (Re<psi,G> / Re<psi,psi_sob>) psi_sob  (Project_Sobolev_Gradient)
__global__ void sob_proj_kernel(double2 *g, const double2 *ps, const SobDev *d, int comp, int64_t n) {
  const double fak = d->q[comp][0] / d->q[comp][1];
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    double2 v = g[l];
    const double2 u = ps[l];
    v.x -= fak * u.x;
    v.y -= fak * u.y;
    g[l] = v;
  }
}

// Residual, particle numbers and the renormalisation decision of one
// iteration (Compute_res, Renormalize_All_Psi), and whether it updates psi.
__global__ void sob_scalars_kernel(SobDev *d, double ar, int ncomp) {
  d->active = (!d->done && d->iters < d->max_iter) ? 1 : 0;
  if (!d->active) return;
  double res = 0;
  bool renorm = false;
  for (int i = 0; i < ncomp; i++) {
    const double q = d->g2[i] * ar;
    res += q * q;
    d->N[i] = ar * d->q[i][2];
    if (fabs(d->N[i] - 1) > 1e-5) renorm = true;
  }
  res = sqrt(res);
  for (int i = 0; i < ncomp; i++) d->scale[i] = renorm ? 1.0 / sqrt(d->N[i]) : 1.0;
  d->res = res;
  d->iters++;
  d->stop = (res > d->eps) ? 0 : 1;
}

// psi <- psi * scale - stepsize G for an active iteration.
__global__ void sob_update_kernel(double2 *psi, const double2 *g, double step, const SobDev *d, int comp, int64_t n) {
  if (!d->active) return;
  const double f = d->scale[comp];
  const bool sc = (f != 1.0);
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < n; l += (int64_t)gridDim.x * blockDim.x) {
    double2 v = psi[l];
    if (sc) {
      v.x *= f;
      v.y *= f;
    }
    const double2 u = g[l];
    v.x -= step * u.x;
    v.y -= step * u.y;
    psi[l] = v;
  }
}

__global__ void sob_commit_kernel(SobDev *d) {
  if (d->active && d->stop) d->done = 1;
}

}  // namespace atus

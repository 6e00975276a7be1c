// ctx.h -- the engine context shared by the host translation units.
#pragma once
#include <cmath>
#include <cuda_runtime.h>

#include <string>

#include "../../include/atus_gpu.h"
#include "kernels.cuh"

using namespace atus;

struct atus_ctx {
  int dim = 0, ncomp = 0, prec = 0;
  int64_t n[3] = {1, 1, 1};
  int lg[3] = {0, 0, 0};
  int64_t npts = 0;
  double d[3] = {0, 0, 0}, dk[3] = {0, 0, 0};
  double ar = 0, ar_k = 0, t = 0, dt = 0.001;
  double alpha[MAXC][3] = {};
  double gs[MAXC * MAXC] = {};  // padded [i*MAXC + j]
  atus_laser laser = {};
  atus_laser laser2 = {};       // second species (two-species programs)
  double win_t0 = 0;            // pulse windows of the two-species bragg_ad:
  double win_dur[2] = {HUGE_VAL, HUGE_VAL};  // species s on while t1 - win_t0 <= win_dur[s]
  size_t csize = 16;            // bytes per complex value
  void *psi[MAXC] = {};
  double *V[MAXC] = {};
  void *scratch = nullptr;      // N complex128 (FP64 staging / spectra)
  void *tw = nullptr;           // twiddles in the field precision
  void *tw64 = nullptr;         // FP64 twiddles (spectra of the FP64 scratch buffer)
  double2 *kt[2][MAXC][3] = {}; // kinetic phase factors [half=0/full=1][comp][axis], FP64
  double *red_partial = nullptr, *red_out = nullptr, *h_red = nullptr;
  cudaStream_t own_stream = nullptr, stream = nullptr;
  int64_t launches = 0;
  bool use_pass2 = true;        // register-staged passes for pencils of 32..256 points
  bool use_cluster1d = true;    // 1D blocks of 2048..8192 points on a 16-CTA cluster
  bool use_tma = false;         // strided 256-point passes fed by TMA tile copies
  int *err_dev = nullptr;       // device error word of bounded waits (0: none)
  bool err_armed = false;       // a kernel that can set it ran since the last check
  long wait_limit = 1L << 22;   // TMA tile waits: try_wait rounds (atus_set_wait_limits)
  int drop_copies = 0;          // TMA passes issue no copies (error-path tests)
  int bragg_stable = 0;         // FP64 Bragg step in the eigenvalue-free form
  std::string err;
  // Sobolev state
  bool sob_ready = false;
  void *sob_lap[MAXC] = {}, *sob_psi[MAXC] = {}, *sob_grad[MAXC] = {};
  double sob_alpha[MAXC] = {};
  double stepsize = 0;
  void *sob_dev = nullptr;              // SobDev in device memory
  cudaGraphExec_t sob_graph = nullptr;  // a chunk of device-side iterations
  double sob_graph_step = 0;            // stepsize the graph was captured with
  void *h_sob = nullptr;                // pinned host copy of the SobDev
  // 1D fields longer than the longest pass (four-step transforms): the field
  // viewed as fs_n1 x fs_n2 (n = fs_n2 * n1 + n2), W_N^m for m < N, and a
  // second N-point FP64 buffer for reordering spectra into natural k order
  int64_t fs_n1 = 0, fs_n2 = 0;
  double2 *fs_tw = nullptr;
  void *fs_tmp = nullptr;
  // asynchronous output snapshots
  void *snap = nullptr;                 // ncomp x N complex128 staging copy
  cudaStream_t copy_stream = nullptr;   // its device->host copies
  cudaEvent_t snap_taken = nullptr;     // the staging copy is complete
  cudaEvent_t snap_read = nullptr;      // the last host copy from it is complete
};

// ------------------------------------------------------------------ errors
static inline int fail(atus_ctx *c, int code, const std::string &msg) {
  if (c) c->err = msg;
  return code;
}
static inline int cuda_check(atus_ctx *c, cudaError_t e, const char *what) {
  if (e == cudaSuccess) return ATUS_OK;
  return fail(c, ATUS_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                           \
  do {                                                     \
    int _r = cuda_check(ctx, (call), #call);               \
    if (_r != ATUS_OK) return _r;                          \
  } while (0)
#define LAUNCHED(ctx)                                                     \
  do {                                                                    \
    (ctx)->launches++;                                                    \
    int _r = cuda_check((ctx), cudaGetLastError(), "kernel launch");      \
    if (_r != ATUS_OK) return _r;                                         \
  } while (0)


static inline Geo geo(const atus_ctx *ctx) {
  Geo g;
  for (int a = 0; a < 3; a++) g.lg[a] = ctx->lg[a];
  g.npts = ctx->npts;
  return g;
}


// guess.cu -- the learned initial guess of the Sobolev ground-state solver.
//
// A small MLP maps the trap and interaction parameters of a ground-state
// problem, (omega_y, omega_z, log g) scaled to O(1), to the 64 coefficients of
// the state in a tensor basis of even Hermite functions (4 per axis).  The
// network trains on ground states that the plain Sobolev descent produced,
// with the kernels below (FP64 throughout: the network is tiny and exact
// gradients make the comparison with the CPU restatement tight):
//
//   guess_grad_kernel     one CTA per sample, one thread per neuron: forward
//                         pass, squared-error loss, backward pass, per-sample
//                         parameter gradients
//   guess_sum_kernel      sums the per-sample gradients in sample order
//   guess_adam_kernel     Adam update
//   guess_fwd_kernel      inference
//   guess_decode_kernel   the coefficients -> the state on the context's grid
//
// Layout of the parameter vector (GUESS_NPARAM doubles): W1[64][3], b1[64],
// W2[64][64], b2[64], W3[64][64], b3[64]; hidden activations tanh, linear
// output.  Loss: mean over samples and outputs of (out - target)^2.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/atus_gpu.h"
#include "ctx.h"

namespace {

constexpr int NI = ATUS_GUESS_NIN, NH = 64, NO = ATUS_GUESS_NOUT, NP = ATUS_GUESS_NPARAM;
static_assert(NH * NI + NH + NH * NH + NH + NO * NH + NO == NP, "parameter layout");
static_assert(NO == NH, "one thread per neuron in every layer");

struct Layout {
  const double *W1, *b1, *W2, *b2, *W3, *b3;
};
__device__ __forceinline__ Layout layout(const double *p) {
  Layout L;
  L.W1 = p;
  L.b1 = L.W1 + NH * NI;
  L.W2 = L.b1 + NH;
  L.b2 = L.W2 + NH * NH;
  L.W3 = L.b2 + NH;
  L.b3 = L.W3 + NO * NH;
  return L;
}

// Forward pass of sample blockIdx.x; leaves h1, h2 in shared memory and
// returns this thread's output.
__device__ __forceinline__ double forward(const Layout &L, const double *x, double *h1, double *h2) {
  const int t = threadIdx.x;
  double a = L.b1[t];
  for (int k = 0; k < NI; k++) a += L.W1[t * NI + k] * x[k];
  h1[t] = tanh(a);
  __syncthreads();
  a = L.b2[t];
  for (int k = 0; k < NH; k++) a += L.W2[t * NH + k] * h1[k];
  h2[t] = tanh(a);
  __syncthreads();
  a = L.b3[t];
  for (int k = 0; k < NH; k++) a += L.W3[t * NH + k] * h2[k];
  return a;
}

__global__ void __launch_bounds__(NH) guess_grad_kernel(const double *p, const double *X, const double *Y, int B,
                                                        double *gpart, double *lpart) {
  __shared__ double x[NI], h1[NH], h2[NH], d3[NH], d2[NH], red[NH];
  const int b = blockIdx.x, t = threadIdx.x;
  const Layout L = layout(p);
  if (t < NI) x[t] = X[(int64_t)b * NI + t];
  __syncthreads();
  const double out = forward(L, x, h1, h2);
  const double sc = 1.0 / ((double)B * NO);
  const double r = out - Y[(int64_t)b * NO + t];
  red[t] = r * r * sc;
  d3[t] = 2.0 * r * sc;
  __syncthreads();
  for (int w = NH / 2; w > 0; w >>= 1) {
    if (t < w) red[t] += red[t + w];
    __syncthreads();
  }
  if (t == 0) lpart[b] = red[0];
  double *g = gpart + (int64_t)b * NP;
  double *gW1 = g, *gb1 = gW1 + NH * NI, *gW2 = gb1 + NH, *gb2 = gW2 + NH * NH, *gW3 = gb2 + NH, *gb3 = gW3 + NO * NH;
  for (int k = 0; k < NH; k++) gW3[t * NH + k] = d3[t] * h2[k];
  gb3[t] = d3[t];
  double a = 0;
  for (int j = 0; j < NO; j++) a += L.W3[j * NH + t] * d3[j];
  d2[t] = a * (1.0 - h2[t] * h2[t]);
  __syncthreads();
  for (int k = 0; k < NH; k++) gW2[t * NH + k] = d2[t] * h1[k];
  gb2[t] = d2[t];
  a = 0;
  for (int j = 0; j < NH; j++) a += L.W2[j * NH + t] * d2[j];
  const double d1 = a * (1.0 - h1[t] * h1[t]);
  for (int k = 0; k < NI; k++) gW1[t * NI + k] = d1 * x[k];
  gb1[t] = d1;
}

__global__ void guess_sum_kernel(const double *gpart, const double *lpart, int B, double *grad, double *loss) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < NP) {
    double s = 0;
    for (int b = 0; b < B; b++) s += gpart[(int64_t)b * NP + q];
    grad[q] = s;
  }
  if (q == 0) {
    double s = 0;
    for (int b = 0; b < B; b++) s += lpart[b];
    *loss = s;
  }
}

__global__ void guess_adam_kernel(double *p, double *m, double *v, const double *g, double lr, double b1, double b2,
                                  double eps, double c1, double c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= NP) return;
  const double gq = g[q];
  const double mq = b1 * m[q] + (1.0 - b1) * gq;
  const double vq = b2 * v[q] + (1.0 - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq / c1) / (sqrt(vq / c2) + eps);
}

__global__ void __launch_bounds__(NH) guess_fwd_kernel(const double *p, const double *X, double *Yout) {
  __shared__ double x[NI], h1[NH], h2[NH];
  const int b = blockIdx.x, t = threadIdx.x;
  if (t < NI) x[t] = X[(int64_t)b * NI + t];
  __syncthreads();
  const double out = forward(layout(p), x, h1, h2);
  Yout[(int64_t)b * NO + t] = out;
}

// psi(i, j, k) = sum_{a,b,c} coef[16 a + 4 b + c] bx[a][i] by[b][j] bz[c][k]
__global__ void guess_decode_kernel(double2 *psi, const double *coef, const double *bx, const double *by,
                                    const double *bz, int n0, int n1, int n2) {
  __shared__ double c[NO];
  if (threadIdx.x < NO) c[threadIdx.x] = coef[threadIdx.x];
  __syncthreads();
  const int64_t npts = (int64_t)n0 * n1 * n2;
  for (int64_t l = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; l < npts; l += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(l % n2), j = (int)((l / n2) % n1), i = (int)(l / ((int64_t)n1 * n2));
    double s = 0;
    for (int a = 0; a < 4; a++) {
      double sa = 0;
      for (int b = 0; b < 4; b++) {
        double sb = 0;
        for (int q = 0; q < 4; q++) sb += c[16 * a + 4 * b + q] * bz[q * n2 + k];
        sa += sb * by[b * n1 + j];
      }
      s += sa * bx[a * n0 + i];
    }
    psi[l] = make_double2(s, 0.0);
  }
}

// Deterministic initial parameters: uniform in +-sqrt(6 / (fan_in + fan_out))
// (Glorot), biases zero, from a splitmix64 stream.
uint64_t splitmix(uint64_t &s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Buffers {
  double *p = nullptr, *m = nullptr, *v = nullptr, *X = nullptr, *Y = nullptr, *gpart = nullptr, *lpart = nullptr,
         *grad = nullptr, *loss = nullptr;
  ~Buffers() {
    for (double *q : {p, m, v, X, Y, gpart, lpart, grad, loss}) cudaFree(q);
  }
};

int alloc_all(Buffers &b, int B, bool train) {
  if (cudaMalloc(&b.p, sizeof(double) * NP) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.X, sizeof(double) * NI * B) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.Y, sizeof(double) * NO * B) != cudaSuccess) return ATUS_E_NOMEM;
  if (!train) return ATUS_OK;
  if (cudaMalloc(&b.gpart, sizeof(double) * NP * (size_t)B) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.lpart, sizeof(double) * B) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.grad, sizeof(double) * NP) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.loss, sizeof(double)) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.m, sizeof(double) * NP) != cudaSuccess) return ATUS_E_NOMEM;
  if (cudaMalloc(&b.v, sizeof(double) * NP) != cudaSuccess) return ATUS_E_NOMEM;
  return ATUS_OK;
}

#define GCK(call)                                   \
  do {                                              \
    if ((call) != cudaSuccess) return ATUS_E_CUDA;  \
  } while (0)

// Hermite functions phi_n(x / l) / sqrt(l), n = 0, 2, 4, 6, on the grid of axis ax.
void hermite_rows(const atus_ctx *ctx, int ax, double l, std::vector<double> &out) {
  const int64_t n = ctx->n[ax];
  out.assign(4 * n, 0.0);
  const double c0 = pow(M_PI, -0.25) / sqrt(l);
  for (int64_t i = 0; i < n; i++) {
    const double x = (double)(i - n / 2) * ctx->d[ax];
    const double u = x / l;
    double pm = 0.0, pc = c0 * exp(-0.5 * u * u);
    for (int q = 0; q <= 6; q++) {
      if (q % 2 == 0) out[(q / 2) * n + i] = pc;
      const double pn = sqrt(2.0 / (q + 1)) * u * pc - sqrt((double)q / (q + 1)) * pm;
      pm = pc;
      pc = pn;
    }
  }
}

}  // namespace

extern "C" {

int atus_guess_init(uint64_t seed, double *params) {
  if (!params) return ATUS_E_ARG;
  uint64_t s = seed;
  auto uni = [&](double a) { return a * (2.0 * (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0) - 1.0); };
  double *W1 = params, *b1 = W1 + NH * NI, *W2 = b1 + NH, *b2 = W2 + NH * NH, *W3 = b2 + NH, *b3 = W3 + NO * NH;
  const double a1 = sqrt(6.0 / (NI + NH)), a2 = sqrt(6.0 / (NH + NH)), a3 = sqrt(6.0 / (NH + NO));
  for (int q = 0; q < NH * NI; q++) W1[q] = uni(a1);
  for (int q = 0; q < NH * NH; q++) W2[q] = uni(a2);
  for (int q = 0; q < NO * NH; q++) W3[q] = uni(a3);
  for (int q = 0; q < NH; q++) b1[q] = b2[q] = 0.0;
  for (int q = 0; q < NO; q++) b3[q] = 0.0;
  return ATUS_OK;
}

int atus_guess_grad(const double *params, const double *X, const double *Y, int B, double *loss, double *grad) {
  if (!params || !X || !Y || B < 1 || !loss || !grad) return ATUS_E_ARG;
  Buffers b;
  int r = alloc_all(b, B, true);
  if (r != ATUS_OK) return r;
  GCK(cudaMemcpy(b.p, params, sizeof(double) * NP, cudaMemcpyHostToDevice));
  GCK(cudaMemcpy(b.X, X, sizeof(double) * NI * B, cudaMemcpyHostToDevice));
  GCK(cudaMemcpy(b.Y, Y, sizeof(double) * NO * B, cudaMemcpyHostToDevice));
  guess_grad_kernel<<<B, NH>>>(b.p, b.X, b.Y, B, b.gpart, b.lpart);
  guess_sum_kernel<<<(NP + 255) / 256, 256>>>(b.gpart, b.lpart, B, b.grad, b.loss);
  GCK(cudaGetLastError());
  GCK(cudaMemcpy(grad, b.grad, sizeof(double) * NP, cudaMemcpyDeviceToHost));
  GCK(cudaMemcpy(loss, b.loss, sizeof(double), cudaMemcpyDeviceToHost));
  return ATUS_OK;
}

int atus_guess_train(double *params, const double *X, const double *Y, int B, int epochs, double lr,
                     double *loss_history) {
  if (!params || !X || !Y || B < 1 || epochs < 1 || !(lr > 0)) return ATUS_E_ARG;
  Buffers b;
  int r = alloc_all(b, B, true);
  if (r != ATUS_OK) return r;
  GCK(cudaMemcpy(b.p, params, sizeof(double) * NP, cudaMemcpyHostToDevice));
  GCK(cudaMemcpy(b.X, X, sizeof(double) * NI * B, cudaMemcpyHostToDevice));
  GCK(cudaMemcpy(b.Y, Y, sizeof(double) * NO * B, cudaMemcpyHostToDevice));
  GCK(cudaMemset(b.m, 0, sizeof(double) * NP));
  GCK(cudaMemset(b.v, 0, sizeof(double) * NP));
  const double b1 = 0.9, b2 = 0.999, eps = 1e-12;
  double c1 = 1.0, c2 = 1.0;
  std::vector<double> hist(epochs);
  double *dhist = nullptr;
  GCK(cudaMalloc(&dhist, sizeof(double) * epochs));
  for (int e = 0; e < epochs; e++) {
    c1 *= b1;
    c2 *= b2;
    guess_grad_kernel<<<B, NH>>>(b.p, b.X, b.Y, B, b.gpart, b.lpart);
    guess_sum_kernel<<<(NP + 255) / 256, 256>>>(b.gpart, b.lpart, B, b.grad, dhist + e);
    guess_adam_kernel<<<(NP + 255) / 256, 256>>>(b.p, b.m, b.v, b.grad, lr, b1, b2, eps, 1.0 - c1, 1.0 - c2);
  }
  cudaError_t ce = cudaGetLastError();
  if (ce == cudaSuccess) ce = cudaMemcpy(params, b.p, sizeof(double) * NP, cudaMemcpyDeviceToHost);
  if (ce == cudaSuccess && loss_history) ce = cudaMemcpy(loss_history, dhist, sizeof(double) * epochs, cudaMemcpyDeviceToHost);
  cudaFree(dhist);
  return ce == cudaSuccess ? ATUS_OK : ATUS_E_CUDA;
}

int atus_guess_predict(const double *params, const double *X, int B, double *coef) {
  if (!params || !X || B < 1 || !coef) return ATUS_E_ARG;
  Buffers b;
  int r = alloc_all(b, B, false);
  if (r != ATUS_OK) return r;
  GCK(cudaMemcpy(b.p, params, sizeof(double) * NP, cudaMemcpyHostToDevice));
  GCK(cudaMemcpy(b.X, X, sizeof(double) * NI * B, cudaMemcpyHostToDevice));
  guess_fwd_kernel<<<B, NH>>>(b.p, b.X, b.Y);
  GCK(cudaGetLastError());
  GCK(cudaMemcpy(coef, b.Y, sizeof(double) * NO * B, cudaMemcpyDeviceToHost));
  return ATUS_OK;
}

int atus_guess_decode(atus_ctx *ctx, int comp, const double *coef, const double *scale) {
  if (!ctx || !coef || !scale || comp < 0 || comp >= ctx->ncomp) return ATUS_E_ARG;
  if (ctx->dim != 3 || ctx->prec != ATUS_PREC_FP64) return fail(ctx, ATUS_E_UNSUPPORTED, "the guess decoder fills 3D FP64 fields");
  std::vector<double> rows[3];
  for (int ax = 0; ax < 3; ax++) {
    if (!(scale[ax] > 0)) return fail(ctx, ATUS_E_ARG, "basis scales must be positive");
    hermite_rows(ctx, ax, scale[ax], rows[ax]);
  }
  double *d = nullptr;
  const size_t nrow = 4 * (ctx->n[0] + ctx->n[1] + ctx->n[2]);
  CK(cudaMalloc(&d, sizeof(double) * (nrow + NO)));
  double *bx = d, *by = bx + 4 * ctx->n[0], *bz = by + 4 * ctx->n[1], *dc = bz + 4 * ctx->n[2];
  cudaError_t e = cudaMemcpyAsync(bx, rows[0].data(), sizeof(double) * rows[0].size(), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(by, rows[1].data(), sizeof(double) * rows[1].size(), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bz, rows[2].data(), sizeof(double) * rows[2].size(), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dc, coef, sizeof(double) * NO, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    guess_decode_kernel<<<148 * 8, 256, 0, ctx->stream>>>((double2 *)ctx->psi[comp], dc, bx, by, bz, (int)ctx->n[0],
                                                         (int)ctx->n[1], (int)ctx->n[2]);
    ctx->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  return cuda_check(ctx, e, "guess decode");
}

}  // extern "C"

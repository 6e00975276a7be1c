// Batched 1D Strang-block kernels, double fields: every (length, threads,
// resident components) combination the autotuner may pick.
#include "batch.cuh"

using namespace atus;

template <int N, int NT, int RES>
static bool k1(BKernel *k) {
  k->fn = (const void *)batch1d_kernel<double, N, NT, RES>;
  k->nt = NT;
  k->smem = sizeof(cplx<double>) * Pad<N>::NP * RES;
  k->B = 0;
  return true;
}

bool batch1d_info_d(int N, int NT, int RES, BKernel *k) {
  if (N == 1024 && NT == 256 && RES == 2) return k1<1024, 256, 2>(k);
  if (N == 1024 && NT == 256 && RES == 1) return k1<1024, 256, 1>(k);
  if (N == 2048 && NT == 256 && RES == 2) return k1<2048, 256, 2>(k);
  if (N == 2048 && NT == 256 && RES == 1) return k1<2048, 256, 1>(k);
  if (N == 4096 && NT == 256 && RES == 2) return k1<4096, 256, 2>(k);
  if (N == 4096 && NT == 256 && RES == 1) return k1<4096, 256, 1>(k);
  if (N == 8192 && NT == 256 && RES == 1) return k1<8192, 256, 1>(k);
  return false;
}

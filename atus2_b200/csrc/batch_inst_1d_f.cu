// Batched 1D Strang-block kernels, float fields: every (length, threads,
// resident components) combination the autotuner may pick.
#include "batch.cuh"

using namespace atus;

template <int N, int NT, int RES>
static bool k1(BKernel *k) {
  k->fn = (const void *)batch1d_kernel<float, N, NT, RES>;
  k->nt = NT;
  k->smem = sizeof(cplx<float>) * Pad<N>::NP * RES;
  k->B = 0;
  return true;
}

bool batch1d_info_f(int N, int NT, int RES, BKernel *k) {
  if (N == 1024 && NT == 256 && RES == 2) return k1<1024, 256, 2>(k);
  if (N == 1024 && NT == 256 && RES == 1) return k1<1024, 256, 1>(k);
  if (N == 1024 && NT == 512 && RES == 2) return k1<1024, 512, 2>(k);
  if (N == 1024 && NT == 512 && RES == 1) return k1<1024, 512, 1>(k);
  if (N == 2048 && NT == 256 && RES == 2) return k1<2048, 256, 2>(k);
  if (N == 2048 && NT == 256 && RES == 1) return k1<2048, 256, 1>(k);
  if (N == 2048 && NT == 512 && RES == 2) return k1<2048, 512, 2>(k);
  if (N == 2048 && NT == 512 && RES == 1) return k1<2048, 512, 1>(k);
  if (N == 4096 && NT == 256 && RES == 2) return k1<4096, 256, 2>(k);
  if (N == 4096 && NT == 256 && RES == 1) return k1<4096, 256, 1>(k);
  if (N == 4096 && NT == 512 && RES == 2) return k1<4096, 512, 2>(k);
  if (N == 4096 && NT == 512 && RES == 1) return k1<4096, 512, 1>(k);
  if (N == 8192 && NT == 256 && RES == 2) return k1<8192, 256, 2>(k);
  if (N == 8192 && NT == 256 && RES == 1) return k1<8192, 256, 1>(k);
  if (N == 8192 && NT == 512 && RES == 2) return k1<8192, 512, 2>(k);
  if (N == 8192 && NT == 512 && RES == 1) return k1<8192, 512, 1>(k);
  if (N == 16384 && NT == 256 && RES == 1) return k1<16384, 256, 1>(k);
  if (N == 16384 && NT == 512 && RES == 1) return k1<16384, 512, 1>(k);
  return false;
}

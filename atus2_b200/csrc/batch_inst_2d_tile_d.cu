// Batched 2D shared-memory tile passes, double fields.
#include "batch.cuh"

using namespace atus;

template <int N, int TC, int MODE>
static bool kt(BKernel *k) {
  using Cfg = BTileCfg<double, N, TC>;
  k->fn = (const void *)batch_tile_kernel<double, N, TC, MODE>;
  k->nt = Cfg::NT;
  k->smem = Cfg::smem;
  k->B = Cfg::B;
  return true;
}

bool batch2d_tile_info_d(int N, int mode, BKernel *k) {
  if (N == 64) {
    if (mode == M2_FWD) return kt<64, 1, M2_FWD>(k);
    if (mode == M2_INV) return kt<64, 1, M2_INV>(k);
    if (mode == M2_KIN) return kt<64, 1, M2_KIN>(k);
    if (mode == M2_NL) return kt<64, 2, M2_NL>(k);
  }
  if (N == 128) {
    if (mode == M2_FWD) return kt<128, 1, M2_FWD>(k);
    if (mode == M2_INV) return kt<128, 1, M2_INV>(k);
    if (mode == M2_KIN) return kt<128, 1, M2_KIN>(k);
    if (mode == M2_NL) return kt<128, 2, M2_NL>(k);
  }
  if (N == 256) {
    if (mode == M2_FWD) return kt<256, 1, M2_FWD>(k);
    if (mode == M2_INV) return kt<256, 1, M2_INV>(k);
    if (mode == M2_KIN) return kt<256, 1, M2_KIN>(k);
    if (mode == M2_NL) return kt<256, 2, M2_NL>(k);
  }
  if (N == 512) {
    if (mode == M2_FWD) return kt<512, 1, M2_FWD>(k);
    if (mode == M2_INV) return kt<512, 1, M2_INV>(k);
    if (mode == M2_KIN) return kt<512, 1, M2_KIN>(k);
    if (mode == M2_NL) return kt<512, 2, M2_NL>(k);
  }
  return false;
}

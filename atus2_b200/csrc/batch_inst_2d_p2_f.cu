// Batched 2D register-staged passes, float fields.
#include "batch.cuh"

using namespace atus;

template <int N, int TC, int MODE, bool STRIDED>
static bool kp(BKernel *k) {
  using Cfg = P2Cfg<float, N, TC>;
  k->fn = (const void *)batch_pass2_kernel<float, N, TC, MODE, STRIDED>;
  k->nt = Cfg::NT;
  k->smem = Cfg::smem;
  k->B = Cfg::B;
  return true;
}

bool batch2d_p2_info_f(int N, int mode, BKernel *k) {
  if (N == 64) {
    if (mode == M2_FWD) return kp<64, 1, M2_FWD, false>(k);
    if (mode == M2_INV) return kp<64, 1, M2_INV, false>(k);
    if (mode == M2_KIN) return kp<64, 1, M2_KIN, true>(k);
    if (mode == M2_NL) return kp<64, 2, M2_NL, false>(k);
  }
  if (N == 128) {
    if (mode == M2_FWD) return kp<128, 1, M2_FWD, false>(k);
    if (mode == M2_INV) return kp<128, 1, M2_INV, false>(k);
    if (mode == M2_KIN) return kp<128, 1, M2_KIN, true>(k);
    if (mode == M2_NL) return kp<128, 2, M2_NL, false>(k);
  }
  if (N == 256) {
    if (mode == M2_FWD) return kp<256, 1, M2_FWD, false>(k);
    if (mode == M2_INV) return kp<256, 1, M2_INV, false>(k);
    if (mode == M2_KIN) return kp<256, 1, M2_KIN, true>(k);
    if (mode == M2_NL) return kp<256, 2, M2_NL, false>(k);
  }
  return false;
}

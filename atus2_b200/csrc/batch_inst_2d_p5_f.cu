// Batched 2D register-staged passes for 512-point pencils, float fields.
#include "batch.cuh"

using namespace atus;

template <int TC, int MODE, bool STRIDED>
static bool k5(BKernel *k) {
  using Cfg = P5Cfg<float, TC>;
  k->fn = (const void *)batch_pass512_kernel<float, TC, MODE, STRIDED>;
  k->nt = Cfg::NT;
  k->smem = Cfg::smem;
  k->B = Cfg::B;
  return true;
}

bool batch2d_p5_info_f(int N, int mode, BKernel *k) {
  if (N != 512) return false;
  if (mode == M2_FWD) return k5<1, M2_FWD, false>(k);
  if (mode == M2_INV) return k5<1, M2_INV, false>(k);
  if (mode == M2_KIN) return k5<1, M2_KIN, true>(k);
  if (mode == M2_NL) return k5<2, M2_NL, false>(k);
  return false;
}

// Register-staged single-transform passes, float fields.
#include "launch.cuh"

int launch_pass2_f_t(atus_ctx *ctx, PassArgs &a, int axis, int mode, bool strided) {
  if (mode == M2_FWD) {
    return strided ? launch_pass2_n<float, 1, M2_FWD, true>(ctx, a, axis) : launch_pass2_n<float, 1, M2_FWD, false>(ctx, a, axis);
  }
  if (mode == M2_INV) {
    return strided ? launch_pass2_n<float, 1, M2_INV, true>(ctx, a, axis) : launch_pass2_n<float, 1, M2_INV, false>(ctx, a, axis);
  }
  return ATUS_E_UNSUPPORTED;
}

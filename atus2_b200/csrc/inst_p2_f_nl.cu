// Register-staged IFFT -> potential step -> FFT passes, float fields.
#include "launch.cuh"

int launch_pass2_f_nl(atus_ctx *ctx, PassArgs &a, int axis, int tc) {
  if (tc == 1) return launch_pass2_n<float, 1, M2_NL, false>(ctx, a, axis);
  if (tc == 2) return launch_pass2_n<float, 2, M2_NL, false>(ctx, a, axis);
  return ATUS_E_UNSUPPORTED;
}

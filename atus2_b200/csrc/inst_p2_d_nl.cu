// Register-staged IFFT -> potential step -> FFT passes, double fields.
#include "launch.cuh"

int launch_pass2_d_nl(atus_ctx *ctx, PassArgs &a, int axis, int tc) {
  if (tc == 1) return launch_pass2_n<double, 1, M2_NL, false>(ctx, a, axis);
  if (tc == 2) return launch_pass2_n<double, 2, M2_NL, false>(ctx, a, axis);
  return ATUS_E_UNSUPPORTED;
}

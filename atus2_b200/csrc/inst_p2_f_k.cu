// Register-staged FFT -> kinetic phase / Sobolev filter -> IFFT passes, float fields.
#include "launch.cuh"

int launch_pass2_f_k(atus_ctx *ctx, PassArgs &a, int axis) {
  return launch_pass2_n<float, 1, M2_KIN, true>(ctx, a, axis);
}

// Register-staged FFT -> kinetic phase / Sobolev filter -> IFFT passes, double fields.
#include "launch.cuh"

int launch_pass2_d_k(atus_ctx *ctx, PassArgs &a, int axis) {
  return launch_pass2_n<double, 1, M2_KIN, true>(ctx, a, axis);
}

// Register-staged FFT -> kinetic phase -> IFFT passes that also sum the Rabi
// balls (the last kinetic pass of a block), float fields.
#include "launch.cuh"

int launch_pass2_f_kr(atus_ctx *ctx, PassArgs &a, int axis) {
  return launch_pass2_n<float, 1, M2_KIN_RABI, true>(ctx, a, axis);
}

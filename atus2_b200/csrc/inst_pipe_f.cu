// Plane pipeline of the 3D real-space half step, float fields.
#include "launch.cuh"

int launch_pipe_f(atus_ctx *ctx, PipeArgs &a, int tc) {
  if (tc == 1) return launch_pipe_n<float, 1>(ctx, a);
  if (tc == 2) return launch_pipe_n<float, 2>(ctx, a);
  return ATUS_E_UNSUPPORTED;
}

// Pass-kernel instantiations: float fields, 1 component(s) per tile.
#include "launch.cuh"

int launch_pass_f1(atus_ctx *ctx, PassArgs &a, int axis) { return launch_pass_n<float, 1>(ctx, a, axis); }

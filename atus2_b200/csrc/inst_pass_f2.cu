// Pass-kernel instantiations: float fields, 2 component(s) per tile.
#include "launch.cuh"

int launch_pass_f2(atus_ctx *ctx, PassArgs &a, int axis) { return launch_pass_n<float, 2>(ctx, a, axis); }

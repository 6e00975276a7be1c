// Pass-kernel instantiations: double fields, 1 component(s) per tile.
#include "launch.cuh"

int launch_pass_d1(atus_ctx *ctx, PassArgs &a, int axis) { return launch_pass_n<double, 1>(ctx, a, axis); }

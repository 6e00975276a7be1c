// Pass-kernel instantiations: double fields, 2 component(s) per tile.
#include "launch.cuh"

int launch_pass_d2(atus_ctx *ctx, PassArgs &a, int axis) { return launch_pass_n<double, 2>(ctx, a, axis); }

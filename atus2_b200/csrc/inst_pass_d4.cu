// Pass-kernel instantiations: double fields, 4 component(s) per tile.
#include "launch.cuh"

int launch_pass_d4(atus_ctx *ctx, PassArgs &a, int axis) { return launch_pass_n<double, 4>(ctx, a, axis); }

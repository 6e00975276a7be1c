// Pass-kernel instantiations: float fields, 4 component(s) per tile.
#include "launch.cuh"

int launch_pass_f4(atus_ctx *ctx, PassArgs &a, int axis) { return launch_pass_n<float, 4>(ctx, a, axis); }

// 1D resident Strang-block instantiations: double fields, 2 component(s).
#include "launch.cuh"

int launch_block1d_d2(atus_ctx *ctx, Block1DArgs &a) { return launch_block1d_n<double, 2>(ctx, a); }

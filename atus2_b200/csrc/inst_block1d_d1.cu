// 1D resident Strang-block instantiations: double fields, 1 component(s).
#include "launch.cuh"

int launch_block1d_d1(atus_ctx *ctx, Block1DArgs &a) { return launch_block1d_n<double, 1>(ctx, a); }

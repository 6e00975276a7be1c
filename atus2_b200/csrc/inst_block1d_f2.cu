// 1D resident Strang-block instantiations: float fields, 2 component(s).
#include "launch.cuh"

int launch_block1d_f2(atus_ctx *ctx, Block1DArgs &a) { return launch_block1d_n<float, 2>(ctx, a); }

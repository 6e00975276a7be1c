// 1D resident Strang-block instantiations: float fields, 1 component(s).
#include "launch.cuh"

int launch_block1d_f1(atus_ctx *ctx, Block1DArgs &a) { return launch_block1d_n<float, 1>(ctx, a); }

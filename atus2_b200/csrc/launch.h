// launch.h -- exported launchers, one per precision and tile component count.
#pragma once
#include "ctx.h"
#include "slab.cuh"

int launch_pass_d1(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass_d2(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass_d4(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass_f1(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass_f2(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass_f4(atus_ctx *ctx, PassArgs &a, int axis);
int launch_block1d_d1(atus_ctx *ctx, Block1DArgs &a);
int launch_block1d_d2(atus_ctx *ctx, Block1DArgs &a);
int launch_block1d_f1(atus_ctx *ctx, Block1DArgs &a);
int launch_block1d_f2(atus_ctx *ctx, Block1DArgs &a);
// Returns ATUS_E_UNSUPPORTED (without touching the fields) when the grid has
// no slab instantiation or the cluster cannot be scheduled.
int launch_slab_d(atus_ctx *ctx, atus::SlabArgs &a, int tc);
int launch_slab_f(atus_ctx *ctx, atus::SlabArgs &a, int tc);

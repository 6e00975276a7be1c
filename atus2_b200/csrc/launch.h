// launch.h -- exported launchers, one per precision and tile component count.
#pragma once
#include "ctx.h"

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

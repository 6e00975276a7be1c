// launch.h -- exported launchers, one per precision and tile component count.
#pragma once
#include "ctx.h"
#include "pass2.cuh"

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
// Register-staged passes (pencils of 32..256 points).  _t: one transform
// (mode M2_FWD / M2_INV, strided or contiguous axis); _k: FFT, kinetic or
// Sobolev filter, IFFT along a strided axis; _nl: IFFT, potential step, FFT
// along the contiguous axis with tc components per tile (1 or 2).  All return
// ATUS_E_UNSUPPORTED, with the fields untouched, when they do not apply.
int launch_pass2_d_t(atus_ctx *ctx, PassArgs &a, int axis, int mode, bool strided);
int launch_pass2_f_t(atus_ctx *ctx, PassArgs &a, int axis, int mode, bool strided);
int launch_pass2_d_k(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass2_f_k(atus_ctx *ctx, PassArgs &a, int axis);
// _kr: the _k kinetic pass that also sums the Rabi balls (M2_KIN_RABI)
int launch_pass2_d_kr(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass2_f_kr(atus_ctx *ctx, PassArgs &a, int axis);
int launch_pass2_d_nl(atus_ctx *ctx, PassArgs &a, int axis, int tc);
int launch_pass2_f_nl(atus_ctx *ctx, PassArgs &a, int axis, int tc);

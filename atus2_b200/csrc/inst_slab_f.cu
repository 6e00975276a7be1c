// Cluster slab-pass instantiations for float fields (one or two components).
#include "slab_launch.cuh"

int launch_slab_f(atus_ctx *ctx, SlabArgs &a, int tc) {
  if (tc == 1) return launch_slab_n<float, 1>(ctx, a);
  if (tc == 2) return launch_slab_n<float, 2>(ctx, a);
  return ATUS_E_UNSUPPORTED;
}

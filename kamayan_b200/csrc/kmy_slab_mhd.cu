// Constrained-transport (FP32) instantiations of the z-streamed stage kernel,
// tiles of 16 and 8 rows, compiled with the FP32 stages' approximate
// division and square root.
#include "kmy_slab_launch.cuh"

namespace kmy {
int slab_dispatch_mhd(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const slab::Args<float> &a,
                      int ty, int grid, size_t smem) {
  return ty == 8 ? slab::dispatch_ty<float, 8, true>(c, mc, ml, a, grid, smem)
                 : slab::dispatch_ty<float, 16, true>(c, mc, ml, a, grid, smem);
}
}  // namespace kmy

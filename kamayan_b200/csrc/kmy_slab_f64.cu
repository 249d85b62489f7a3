// FP64 instantiations of the z-streamed stage kernel (tiles of 8 rows: twice
// the FP32 shared memory per cell leaves room for one 256-thread CTA per SM).
#include "kmy_slab_launch.cuh"

namespace kmy {
int slab_dispatch_f64(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const slab::Args<double> &a,
                      int ty, int grid, size_t smem) {
  if (ty != 8) {
    c->err = "the FP64 z-streamed stage runs tiles of 8 rows";
    return KMY_ERR_BAD_PARAM;
  }
  return slab::dispatch_ty<double, 8>(c, mc, ml, a, grid, smem);
}
}  // namespace kmy

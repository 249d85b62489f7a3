// kmy_slab_launch.cuh -- launch of the z-streamed stage kernels of one
// precision (included by kmy_slab_f32.cu and kmy_slab_f64.cu, which compile
// with their precision's flags).
#pragma once

#include <atomic>

#include "../../include/kmy_hydro.h"
#include "kmy_slab.cuh"

namespace kmy {
namespace slab {

constexpr size_t kMaxSmem = 227 * 1024;  // dynamic shared memory per CTA on sm_100

template <typename R, int TY, int RECON, int RIEMANN, bool MHD = false>
int launch_kind(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const Args<R> &a, int grid,
                size_t smem) {
  auto kern = k_slab_stage<R, TY, RECON, RIEMANN, MHD>;
  // the shared-memory opt-in once per device (to the per-CTA maximum, which
  // covers every padded row length), so a stream capture sees launches only
  static std::atomic<unsigned long long> opted{0};
  const unsigned long long bit = c->device < 64 ? 1ull << c->device : 0ull;
  if (smem > kMaxSmem) {
    c->err = "slab stage: shared-memory plan above the per-CTA maximum";
    return KMY_ERR_BAD_PARAM;
  }
  if (!bit || !(opted.load() & bit)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMaxSmem));
    if (e != cudaSuccess) return cuda_check(c, e, "slab smem attribute");
    opted.fetch_or(bit);
  }
  kern<<<unsigned(grid), Tile<TY, R, MHD>::NT, smem, c->stream>>>(mc, ml, a);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "slab stage");
}

template <typename R, int TY, bool MHD = false>
int dispatch_ty(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const Args<R> &a, int grid,
                size_t smem) {
  const int rec = c->prm.recon, rie = c->prm.riemann;
#define KMY_SLAB(RC)                                                                          \
  if (rec == RC)                                                                              \
    return rie == HLL ? launch_kind<R, TY, RC, HLL, MHD>(c, mc, ml, a, grid, smem)            \
                      : launch_kind<R, TY, RC, HLLC, MHD>(c, mc, ml, a, grid, smem);
  KMY_SLAB(FOG)
  KMY_SLAB(PLM)
  KMY_SLAB(PPM)
  KMY_SLAB(WENOZ)
#undef KMY_SLAB
  c->err = "no slab kernel for this reconstruction";
  return KMY_ERR_BAD_PARAM;
}

}  // namespace slab
}  // namespace kmy

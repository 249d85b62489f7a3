// kmy_fused.cu -- host side of the fused RK stage: argument set-up and
// precision dispatch.
#include "../../include/kmy_hydro.h"
#include "kmy_fused.cuh"

namespace kmy {

// +inf as the starting value of the CTA-wide atomic minimum
__global__ void k_reset_dtmin_fused(DevClock *clock) { clock->dtmin_bits = 0x7FF0000000000000ull; }

int fused_dispatch_f64(kmy_ctx *c, FusedArgs<double> a);
int fused_dispatch_f32(kmy_ctx *c, FusedArgs<float> a);

template <typename S>
static FusedArgs<S> fused_args(kmy_ctx *c, Container &base, Container &md0, Container &md1,
                               double beta, bool stored, bool last) {
  FusedArgs<S> a{};
  a.m = c->m;
  a.eos = c->eos;
  a.limiter = c->prm.limiter;
  a.u0 = static_cast<const S *>(md0.cc);
  a.u0lo = static_cast<const float *>(md0.ener_lo);
  a.ub = static_cast<const S *>(base.cc);
  a.ublo = static_cast<const float *>(base.ener_lo);
  a.u1 = static_cast<S *>(md1.cc);
  a.u1lo = static_cast<float *>(md1.ener_lo);
  a.prim = static_cast<const S *>(c->prim);
  // FP32 keeps the primitives of each stage's output for the next stage (its
  // staging then skips the FP64 energy recovery); in FP64 the extra stores
  // cost more than the conversions they save, so every stage converts.
  a.prim_out = sizeof(S) == 4 ? static_cast<S *>(c->prim_alt) : nullptr;
  a.stored = stored ? 1 : 0;
  a.last = last ? 1 : 0;
  a.beta = beta;
  a.clock = c->clock;
  return a;
}

int launch_fused_stage(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta,
                       bool stored, bool last) {
  if (c->prm.mhd) {
    c->err = "fused stage: constrained transport runs through the task kernels";
    return KMY_ERR_BAD_PARAM;
  }
  if (last) {
    k_reset_dtmin_fused<<<1, 1, 0, c->stream>>>(c->clock);
    c->launches++;
  }
  if (c->esz == 8)
    return fused_dispatch_f64(c, fused_args<double>(c, base, md0, md1, beta, stored, last));
  return fused_dispatch_f32(c, fused_args<float>(c, base, md0, md1, beta, stored, last));
}

}  // namespace kmy

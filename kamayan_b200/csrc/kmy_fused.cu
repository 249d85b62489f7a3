// kmy_fused.cu -- host side of the fused RK stage: argument set-up and
// precision dispatch.
#include "../../include/kmy_hydro.h"
#include "kmy_fused.cuh"

namespace kmy {

// +inf as the starting value of the CTA-wide atomic minimum
__global__ void k_reset_dtmin_fused(DevClock *clock) { clock->dtmin_bits = 0x7FF0000000000000ull; }

// Why a context's constrained-transport stage cannot run fused, or null.
// The fused stage reads halos from neighbouring blocks' interiors; the edge
// EMFs' ghost-layer fluxes are copied the same way, which holds for periodic
// and outflow boundaries on a single-level mesh.
const char *fused_ct_unsupported(const kmy_ctx *c) {
  const MeshDesc &m = c->m;
  if (m.ndim < 2) return "constrained transport needs two or more dimensions";
  if (c->amr.on) return "adaptive meshes run the per-task kernels";
  if (c->prm.beta.size() < 2) return "rk1 runs constrained transport through the per-task kernels";
  for (int d = 0; d < m.ndim; d++)
    for (int s = 0; s < 2; s++)
      if (m.bc[d][s] == BC_REFLECT) return "reflecting boundaries with constrained transport";
  return nullptr;
}

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
  if (c->prm.mhd) {
    // constrained transport: the primitives and the time step follow the
    // face update, which runs after this kernel
    a.prim_out = nullptr;
    a.last = 0;
    a.fc0 = static_cast<const S *>(md0.fc);
    a.flux = static_cast<S *>(c->flux);
  }
  return a;
}

int launch_fused_stage(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta,
                       bool stored, bool last) {
  if (c->prm.mhd) {
    if (const char *why = fused_ct_unsupported(c)) {
      c->err = std::string("fused stage: ") + why + "; use the task path";
      return KMY_ERR_BAD_PARAM;
    }
    if (const int rc = ensure_flux(c)) return rc;
    last = false;
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

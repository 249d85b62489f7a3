// FP64 instantiations of the fused stage kernel (separate unit for parallel builds).
// FP64 divisions and square roots by Newton-Raphson refinement (kdiv, ksqrt
// in kmy_device.cuh), as in the z-streamed FP64 stage; -DKMY_F64_NR=0 builds
// IEEE division and square root.
#ifndef KMY_F64_NR
#define KMY_F64_NR 1
#endif
#include "kmy_fused.cuh"

namespace kmy {
int fused_dispatch_f64(kmy_ctx *c, FusedArgs<double> a) { return fused_dispatch<double>(c, a); }
}  // namespace kmy

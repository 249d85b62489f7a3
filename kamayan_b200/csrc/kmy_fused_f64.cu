// FP64 instantiations of the fused stage kernel (separate unit for parallel builds).
#include "kmy_fused.cuh"

namespace kmy {
int fused_dispatch_f64(kmy_ctx *c, FusedArgs<double> a) { return fused_dispatch<double>(c, a); }
}  // namespace kmy

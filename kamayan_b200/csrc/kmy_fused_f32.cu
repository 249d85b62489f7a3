// FP32 instantiations of the fused stage kernel (separate unit for parallel builds).
#include "kmy_fused.cuh"

namespace kmy {
int fused_dispatch_f32(kmy_ctx *c, FusedArgs<float> a) { return fused_dispatch<float>(c, a); }
}  // namespace kmy

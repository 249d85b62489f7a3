// double instantiations of the batched fused stage (separate unit for parallel builds).
// FP64 divisions and square roots by Newton-Raphson refinement (kdiv, ksqrt
// in kmy_device.cuh), as in the z-streamed FP64 stage; -DKMY_F64_NR=0 builds
// IEEE division and square root.
#ifndef KMY_F64_NR
#define KMY_F64_NR 1
#endif
#include "kmy_batch.cuh"

namespace kmy {
int batch_stage_f64(cudaStream_t stream, int ndim, int recon, int riemann, const void *desc,
                   const long long *prefix, const int *n, int stage, int *grid_io) {
  return batch_stage<double>(stream, ndim, recon, riemann, desc, prefix, n, stage, grid_io);
}
int batch_controller_f64(cudaStream_t stream, void *desc, const int *n, int capacity, BatchStatus *st) {
  return batch_controller<double>(stream, desc, n, capacity, st);
}
}  // namespace kmy

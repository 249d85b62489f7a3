// kmy_kat.cu -- the library's device reconstruction functions on a batch of
// stencils, for checking them against known answers.
//
// Each stage kernel reconstructs through its own form of the reference's
// Reconstruct (reconstruction.hpp:11-142); this entry point runs exactly
// those device functions, so the reference's reconstruction unit tests
// (src/physics/hydro/tests/test_reconstruction.cpp:13-194: polynomial
// exactness and left/right mirror symmetry) pin the CUDA code, not only the
// CPU restatement:
//   impl 0  FP64 Reconstruct                   (per-task kernels, k_face_flux)
//   impl 1  FP64 two-division WENO-Z, dividing by Newton-Raphson
//           reciprocals                        (FP64 brick and batched stages)
//   impl 2  FP32 Reconstruct                   (per-lane FP32 path)
//   impl 3  FP32 packed WenoZBoth2 / per lane  (FP32 brick stage)
//   impl 4  FP32 packed WenoZPair / per lane   (z-streamed FP32 stage)
//   impl 5  FP64 ReconPair, lane by lane       (z-streamed FP64 stage: WENO-Z
//                                               divides by Newton-Raphson reciprocals)
//   impl 6  the FP64 stages' Newton-Raphson reciprocal of
//           stencil[0] (out[0]) and square root of stencil[1] (out[1]), for
//           checking against IEEE division and square root
// This unit compiles with the FP32 stage kernels' flags (approximate
// division and square root, denormals flushed), so impls 2-4 round as they do.
#include <string>

#include "../../include/kmy_hydro.h"
#include "kmy_slab.cuh"

namespace kmy {
namespace {

template <int RECON>
__device__ void kat_one(int impl, int limiter, const double *s, double *out) {
  if (impl <= 1) {
    double d[5];
    for (int k = 0; k < 5; k++) d[k] = s[k];
    double vm, vp;
    if (impl == 1 && RECON == WENOZ) WenoZBothTwoDiv<double, DivNR>(d, vm, vp);
    else Reconstruct<RECON, double>(limiter, d, vm, vp);
    out[0] = vm;
    out[1] = vp;
  } else if (impl == 2) {
    float f[5];
    for (int k = 0; k < 5; k++) f[k] = float(s[k]);
    float vm, vp;
    Reconstruct<RECON, float>(limiter, f, vm, vp);
    out[0] = vm;
    out[1] = vp;
  } else if (impl == 6) {
    out[0] = rcp_nr(s[0]);
    out[1] = sqrt_nr(s[1]);
  } else if (impl == 5) {
    double2 f[5];
    for (int k = 0; k < 5; k++) f[k] = make_double2(s[k], s[k]);
    double2 vm, vp;
    slab::ReconPair<RECON>(limiter, f, vm, vp);
    out[0] = vm.x;
    out[1] = vp.x;
    out[2] = (vm.x == vm.y && vp.x == vp.y) ? 0.0 : 1.0;
  } else {
    // both lanes carry the case; lane .y must agree with lane .x
    float2 f[5];
    for (int k = 0; k < 5; k++) f[k] = make_float2(float(s[k]), float(s[k]));
    float2 vm, vp;
    if (impl == 3) ReconstructBoth2<RECON>(limiter, f, vm, vp);
    else slab::ReconPair<RECON>(limiter, f, vm, vp);
    out[0] = vm.x;
    out[1] = vp.x;
    out[2] = (vm.x == vm.y && vp.x == vp.y) ? 0.0 : 1.0;
  }
}

__global__ void k_reconstruct_stencils(int recon, int limiter, int impl, const double *st, int n, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double o[3] = {0.0, 0.0, 0.0};
  const double *s = st + 5 * size_t(i);
  switch (recon) {
    case FOG: kat_one<FOG>(impl, limiter, s, o); break;
    case PLM: kat_one<PLM>(impl, limiter, s, o); break;
    case PPM: kat_one<PPM>(impl, limiter, s, o); break;
    default: kat_one<WENOZ>(impl, limiter, s, o); break;
  }
  for (int k = 0; k < 3; k++) out[3 * size_t(i) + k] = o[k];
}

}  // namespace
}  // namespace kmy

extern "C" int kmy_reconstruct_stencils(const char *reconstruction, const char *slope_limiter, int impl,
                                        const double *stencils, int n, double *out) {
  using namespace kmy;
  if (!reconstruction || !slope_limiter || !stencils || !out || n < 0 || impl < 0 || impl > 6)
    return KMY_ERR_BAD_PARAM;
  const std::string r(reconstruction), l(slope_limiter);
  const int recon = r == "fog" ? FOG : r == "plm" ? PLM : r == "ppm" ? PPM : r == "wenoz" ? WENOZ : -1;
  const int lim = l == "minmod" ? MINMOD : l == "van_leer" ? VAN_LEER : l == "mc" ? MC : -1;
  if (recon < 0 || lim < 0) return KMY_ERR_BAD_PARAM;
  if (n == 0) return KMY_OK;
  double *d_in = nullptr, *d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_in, sizeof(double) * 5 * size_t(n));
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(double) * 3 * size_t(n));
  if (e == cudaSuccess) e = cudaMemcpy(d_in, stencils, sizeof(double) * 5 * size_t(n), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_reconstruct_stencils<<<(n + 127) / 128, 128>>>(recon, lim, impl, d_in, n, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d_out, sizeof(double) * 3 * size_t(n), cudaMemcpyDeviceToHost);
  if (d_in) cudaFree(d_in);
  if (d_out) cudaFree(d_out);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return KMY_ERR_CUDA;
  }
  return KMY_OK;
}

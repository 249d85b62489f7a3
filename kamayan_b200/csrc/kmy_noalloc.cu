// kmy_noalloc.cu -- conserved-variable sums for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc: a host framework that owns every byte
// of device memory through its own pool (a Kokkos/Parthenon memory space or a
// serving process with a fixed memory budget), and code running where an
// allocation is not allowed or would synchronise the whole device (inside a
// stream callback, or between launches of a latency-critical loop).  For them
// kmy_conserved_sums_noalloc works on caller-owned device arrays and keeps its
// per-CTA partial sums in the file-scope device array below instead of
// allocating a buffer.
//
// The array is a fixed, modest size (kNoallocMaxVars x kNoallocCtas pairs of
// doubles, 75.8 KiB) and every GPU that loads this library holds it until the
// process exits.  Its device address is looked up once per CUDA context, on
// the first call made with that context current (a device reset starts a new
// context, which looks it up again).  All calls on a device share it and it keeps the previous
// call's contents: each call overwrites every partial slot it reads, so
// nothing needs clearing, but calls whose kernels overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the
// caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>

#include "../../include/kmy_hydro.h"

namespace kmy {
namespace {

constexpr int kNoallocMaxVars = 8;   // cell conserved components: 5 hydro, 8 with CT
constexpr int kNoallocCtas = 592;    // 4 CTAs per SM on 148 SMs
constexpr int kNoallocThreads = 256;

// (sum, compensation) per (variable, CTA).  Host code must not pass this name
// to a kernel: on the host it is only a stand-in for the device symbol.
__device__ __align__(256) double g_sum_scratch[2 * kNoallocMaxVars * kNoallocCtas];

std::mutex g_setup_mutex;
// Device address of g_sum_scratch per CUDA context (by context id): a device
// reset destroys the primary context and the module is loaded again, possibly
// at another address, in the new context, which then gets its own lookup.
std::map<unsigned long long, double *> g_scratch_dev;

using CtxGetCurrent = CUresult (*)(CUcontext *);
using CtxGetId = CUresult (*)(CUcontext, unsigned long long *);

template <typename F>
F driver_fn(const char *name) {
  void *p = nullptr;
  cudaDriverEntryPointQueryResult q{};
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(p);
}

// Id of the context current on this thread (0 if none is current yet).
unsigned long long current_context_id() {
  static CtxGetCurrent get_current = driver_fn<CtxGetCurrent>("cuCtxGetCurrent");
  static CtxGetId get_id = driver_fn<CtxGetId>("cuCtxGetId");
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Device address of g_sum_scratch in the current context, looked up with
// cudaGetSymbolAddress the first time a context calls (which also makes the
// runtime's context current if it was not yet).
int scratch_address(double **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  unsigned long long id = current_context_id();
  if (id) {
    auto it = g_scratch_dev.find(id);
    if (it != g_scratch_dev.end()) {
      *out = it->second;
      return KMY_OK;
    }
  }
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_sum_scratch);
  if (e != cudaSuccess || !p) {
    std::fprintf(stderr, "kmy_conserved_sums_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
    return KMY_ERR_CUDA;
  }
  if (!id) id = current_context_id();
  if (id) g_scratch_dev[id] = static_cast<double *>(p);
  *out = static_cast<double *>(p);
  return KMY_OK;
}

struct Layout {
  int nb, ncons;
  int np[3], nx[3], g[3];
  long long P;
};

__device__ __forceinline__ void neumaier(double &s, double &c, double x) {
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

// Per-CTA compensated sums over the interior cells, into scratch[(v*CTAs + cta)*2].
__global__ void __launch_bounds__(kNoallocThreads)
k_noalloc_partials(Layout L, const double *cons, double vol, double *scratch) {
  __shared__ double ss[kNoallocThreads], sc[kNoallocThreads];
  const long long per = (long long)L.nx[0] * L.nx[1] * L.nx[2];
  const long long tot = per * L.nb;
  const long long NP = (long long)L.nb * L.P;
  for (int v = 0; v < L.ncons; v++) {
    double s = 0.0, c = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
      const int b = int(t / per);
      long long r = t - (long long)b * per;
      const int i = int(r % L.nx[0]);
      r /= L.nx[0];
      const int j = int(r % L.nx[1]);
      const int k = int(r / L.nx[1]);
      const long long n = (long long)b * L.P +
                          ((long long)(k + L.g[2]) * L.np[1] + (j + L.g[1])) * L.np[0] + (i + L.g[0]);
      neumaier(s, c, cons[v * NP + n] * vol);
    }
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      double S = 0.0, C = 0.0;
      for (int q = 0; q < kNoallocThreads; q++) {
        neumaier(S, C, ss[q]);
        C += sc[q];
      }
      scratch[(v * kNoallocCtas + blockIdx.x) * 2] = S;
      scratch[(v * kNoallocCtas + blockIdx.x) * 2 + 1] = C;
    }
    __syncthreads();
  }
}

// One thread per variable folds the CTA partials in CTA order.
__global__ void k_noalloc_final(int ncons, const double *scratch, double *out) {
  const int v = threadIdx.x;
  if (v >= ncons) return;
  double S = 0.0, C = 0.0;
  for (int q = 0; q < kNoallocCtas; q++) {
    neumaier(S, C, scratch[(v * kNoallocCtas + q) * 2]);
    C += scratch[(v * kNoallocCtas + q) * 2 + 1];
  }
  out[v] = S + C;
}

}  // namespace
}  // namespace kmy

extern "C" int kmy_conserved_sums_noalloc(const double *cons, int ncons, int nblocks,
                                          const int ncells_pad[3], const int nx[3],
                                          const int nghost[3], double cell_volume,
                                          double *out_dev, void *stream) {
  using namespace kmy;
  if (!cons || !out_dev || !ncells_pad || !nx || !nghost || nblocks <= 0) return KMY_ERR_BAD_PARAM;
  if (ncons < 1 || ncons > kNoallocMaxVars) {
    std::fprintf(stderr,
                 "kmy_conserved_sums_noalloc: ncons = %d is outside 1..%d, the size of the "
                 "static scratch array\n", ncons, kNoallocMaxVars);
    return KMY_ERR_BAD_PARAM;
  }
  Layout L{};
  L.nb = nblocks;
  L.ncons = ncons;
  L.P = 1;
  for (int d = 0; d < 3; d++) {
    if (nx[d] < 1 || nghost[d] < 0 || ncells_pad[d] != nx[d] + 2 * nghost[d]) return KMY_ERR_BAD_PARAM;
    L.np[d] = ncells_pad[d];
    L.nx[d] = nx[d];
    L.g[d] = nghost[d];
    L.P *= ncells_pad[d];
  }
  double *scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  k_noalloc_partials<<<kNoallocCtas, kNoallocThreads, 0, s>>>(L, cons, cell_volume, scratch);
  k_noalloc_final<<<1, 32, 0, s>>>(ncons, scratch, out_dev);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "kmy_conserved_sums_noalloc: %s\n", cudaGetErrorString(e));
    return KMY_ERR_CUDA;
  }
  return KMY_OK;
}

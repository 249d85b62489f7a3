// kmy_batch.cuh -- launchers for the batched fused stage (k_fused_batch) and
// the per-solve dt controller of a batch.  One instantiation set per storage
// precision lives in kmy_batch_f64.cu / kmy_batch_f32.cu.
#pragma once

#include "kmy_fused.cuh"

namespace kmy {

// Per-solve status copied to the host after every tick of a batch.
struct BatchStatus {
  int done;
  int status;
  int ncycle;
  int pad;
  double time;
  double dt;
};

// Advance every solve of the batch after its last stage: clock update, step
// limit, reset of the CFL minimum for the next step, and the status copy.
template <typename S>
__global__ void k_batch_controller(SolveDesc<S> *d, const int *nsolves_dev, BatchStatus *st) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= *nsolves_dev) return;
  SolveDesc<S> &q = d[s];
  DevClock *clk = q.clock;
  if (!clk->done) {
    advance_clock(clk, q.tp);
    if (q.nlim >= 0 && clk->ncycle >= q.nlim) clk->done = 1;
    if (clk->status) clk->done = 1;
    clk->dtmin_bits = 0x7FF0000000000000ull;
    q.stored = 0;
  }
  BatchStatus b;
  b.done = clk->done;
  b.status = clk->status;
  b.ncycle = clk->ncycle;
  b.pad = 0;
  b.time = clk->time;
  b.dt = clk->dt;
  st[s] = b;
}

template <typename S, int NDIM, int RECON, int RIEMANN>
static int batch_stage_t(cudaStream_t stream, const void *desc, const long long *prefix, const int *n,
                         int stage, int *grid_io) {
  using Sh = FusedShape<NDIM, RECON>;
  auto kern = k_fused_batch<S, NDIM, RECON, RIEMANN>;
  const size_t smem = Sh::template smem_bytes<S>();
  if (*grid_io <= 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return 5;
    int per_sm = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, Sh::NT, smem);
    if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    *grid_io = per_sm * sms;
  }
  kern<<<*grid_io, Sh::NT, smem, stream>>>(static_cast<const SolveDesc<S> *>(desc), prefix, n, stage);
  return cudaGetLastError() == cudaSuccess ? 0 : 5;
}

template <typename S>
int batch_stage(cudaStream_t stream, int ndim, int recon, int riemann, const void *desc,
                const long long *prefix, const int *n, int stage, int *grid_io) {
#define KMY_BT(ND, RC)                                                                        \
  if (ndim == ND && recon == RC)                                                              \
    return riemann == HLL ? batch_stage_t<S, ND, RC, HLL>(stream, desc, prefix, n, stage, grid_io) \
                          : batch_stage_t<S, ND, RC, HLLC>(stream, desc, prefix, n, stage, grid_io);
#define KMY_BT_ND(ND) KMY_BT(ND, FOG) KMY_BT(ND, PLM) KMY_BT(ND, PPM) KMY_BT(ND, WENOZ)
  KMY_BT_ND(1)
  KMY_BT_ND(2)
  KMY_BT_ND(3)
#undef KMY_BT_ND
#undef KMY_BT
  return 1;
}

template <typename S>
int batch_controller(cudaStream_t stream, void *desc, const int *n, int capacity, BatchStatus *st) {
  k_batch_controller<S><<<(capacity + 127) / 128, 128, 0, stream>>>(static_cast<SolveDesc<S> *>(desc), n, st);
  return cudaGetLastError() == cudaSuccess ? 0 : 5;
}

}  // namespace kmy

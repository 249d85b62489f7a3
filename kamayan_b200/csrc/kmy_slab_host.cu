// kmy_slab_host.cu -- host side of the z-streamed 3D hydro stage
// (kmy_slab.cuh): eligibility, tensor maps over the ghost-padded containers,
// and the persistent launch over the (block, tile) work list.  The kernels of
// each precision live in kmy_slab_f32.cu and kmy_slab_f64.cu.
#include <cudaTypedefs.h>

#include <atomic>
#include <cstring>
#include <mutex>
#include <type_traits>

#include "../../include/kmy_hydro.h"
#include "kmy_slab.cuh"

namespace kmy {

int slab_dispatch_f32(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const slab::Args<float> &a,
                      int ty, int grid, size_t smem);
int slab_dispatch_f64(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const slab::Args<double> &a,
                      int ty, int grid, size_t smem);
int slab_dispatch_mhd(kmy_ctx *c, const CUtensorMap &mc, const CUtensorMap &ml, const slab::Args<float> &a,
                      int ty, int grid, size_t smem);

namespace {

__global__ void k_reset_dtmin_slab(DevClock *clock) { clock->dtmin_bits = 0x7FF0000000000000ull; }

// Padded rows per TMA row group: the group's bytes must be a multiple of 16.
int row_group(int np0, int esz) {
  if ((np0 * esz) % 16 == 0) return 1;
  if ((2 * np0 * esz) % 16 == 0) return 2;
  return 0;
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn(std::string *err) {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  if (!fn && err) *err = "cuTensorMapEncodeTiled is not available from the driver";
  return fn;
}

// Tensor map over one container array of esz-byte values: dims (row group,
// row groups, planes of all blocks [, variables]); the box is one tile's
// staged rows of two planes.  The row group is the context's (its energy low
// words group as its FP32 conserved values do).
int make_map(kmy_ctx *c, CUtensorMap *map, const void *base, int nvar, int staged_rows, int esz) {
  const MeshDesc &m = c->m;
  const int R = row_group(m.np[0], int(c->esz));
  auto fn = encode_fn(&c->err);
  if (!fn) return KMY_ERR_CUDA;
  const cuuint64_t es = cuuint64_t(esz);
  cuuint64_t dims[4] = {cuuint64_t(R) * m.np[0], cuuint64_t(m.np[1] / R), cuuint64_t(m.np[2]) * m.nb,
                        cuuint64_t(nvar)};
  cuuint64_t strides[3] = {cuuint64_t(R) * m.np[0] * es, cuuint64_t(m.np[0]) * m.np[1] * es,
                           cuuint64_t(m.nb) * m.P * es};
  cuuint32_t box[4] = {cuuint32_t(R * m.np[0]), cuuint32_t(staged_rows / R), 2u, cuuint32_t(nvar)};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const cuuint32_t rank = nvar > 1 ? 4 : 3;
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = fn(map, dt, rank, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    c->err = "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")";
    return KMY_ERR_CUDA;
  }
  return KMY_OK;
}

int sm_count(int device) {
  static std::atomic<int> cache[64];
  if (device < 0 || device >= 64) return 148;
  int v = cache[device].load();
  if (v <= 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
    cache[device].store(v);
  }
  return v;
}

// Shared memory of one CTA and CTAs per SM of the plan for this precision and tile.
int slab_smem(const kmy_ctx *c, int ty) {
  const int np0 = c->m.np[0];
  if (c->prm.mhd)
    return ty == 8 ? slab::Smem<8, float, true>(np0).total() : slab::Smem<16, float, true>(np0).total();
  if (c->esz == 4) return ty == 8 ? slab::Smem<8, float>(np0).total() : slab::Smem<16, float>(np0).total();
  return ty == 8 ? slab::Smem<8, double>(np0).total() : slab::Smem<16, double>(np0).total();
}
int slab_ctas(const kmy_ctx *c, int ty) {
  if (c->prm.mhd) return ty == 8 ? slab::Tile<8, float, true>::CTAS : slab::Tile<16, float, true>::CTAS;
  if (c->esz == 4) return ty == 8 ? slab::Tile<8, float>::CTAS : slab::Tile<16, float>::CTAS;
  return ty == 8 ? slab::Tile<8, double>::CTAS : slab::Tile<16, double>::CTAS;
}

}  // namespace

// Rows per tile for this context: the deck's (or the tuner's) choice, else
// in FP32 16 where the block height allows it (measured faster than 8 on the
// 256^3 WENO-Z workload, and 3.54 against 4.56 ms per step on the 192^3
// Orszag-Tang workload with constrained transport), else 8; FP64 runs 8.
int slab_rows(const kmy_ctx *c) {
  if (c->prm.slab_rows) return c->prm.slab_rows;
  if (c->esz == 8) return 8;
  return c->m.nx[1] % 16 == 0 ? 16 : 8;
}

const char *slab_unsupported(const kmy_ctx *c) {
  const MeshDesc &m = c->m;
  if (c->esz != 4 && c->esz != 8) return "the z-streamed stage is FP32 or FP64";
  if (m.ndim != 3) return "the z-streamed stage is 3D";
  if (c->prm.mhd) {
    if (c->esz != 4) return "constrained transport runs the FP64 brick stage";
    // the cell pass of the streamed face update keeps the field's face ghosts
    if (ct_stream_unsupported(c)) return "constrained transport without the streamed face update";
    for (int d = 0; d < 3; d++)
      for (int side = 0; side < 2; side++)
        if (m.bc[d][side] == BC_REFLECT) return "constrained transport with reflecting boundaries";
  }
  if (c->amr.on) return "adaptive meshes run the per-task kernels";
  if (m.nx[0] != slab::NX) return "the z-streamed stage needs 32 cells per block along x";
  const int ty = slab_rows(c);
  if (c->esz == 8 && ty != 8) return "the FP64 z-streamed stage runs tiles of 8 rows";
  if (m.nx[1] % ty != 0) return "the block height is not a multiple of the tile's rows";
  if (m.nx[2] % 2 != 0) return "the z-streamed stage needs an even block size along z";
  for (int d = 0; d < 3; d++)
    if (m.g[d] < slab::HH) return "the z-streamed stage needs 3 or more ghost cells";
  const int R = row_group(m.np[0], int(c->esz));
  if (!R) return "padded rows do not group into 16-byte multiples";
  if ((m.g[1] - slab::HH) % R || (ty + 2 * slab::HH) % R || m.np[1] % R || ty % R)
    return "staged rows do not align with the row groups";
  if ((size_t(m.np[0]) * m.np[1] * 4) % 16) return "padded planes are not a multiple of 16 bytes";
  if ((long long)m.np[2] * m.nb >= (1ll << 31)) return "too many planes for a tensor map";
  if (slab_smem(c, ty) * slab_ctas(c, ty) > 227 * 1024) return "padded rows too long for the shared-memory plan";
  return nullptr;
}

// Whether the z-streamed stage runs this context's stages: where it applies,
// unless the deck asks for the brick stage, and by default (stage_kernel =
// auto) only on meshes with enough (block, tile) work items to fill the GPU.
// A work item walks a whole block along z, one CTA per SM: with fewer items
// than about half the SMs (FP32) or than the SMs (FP64, a slower item) the
// brick stage, which spreads a block over many CTAs, is faster (a 64^3 mesh
// of 32^3 blocks has 16 FP32 items).
bool slab_runs(const kmy_ctx *c) {
  if (c->prm.stage_kernel == 1 || slab_unsupported(c)) return false;
  if (c->prm.stage_kernel != 0) return true;
  const long long items = (long long)c->m.nb * (c->m.nx[1] / slab_rows(c));
  const int sms = sm_count(c->device);
  return c->esz == 8 ? items >= sms : 2 * items >= sms;
}

bool ct_cells_on_slab(const kmy_ctx *c) { return c->prm.mhd && slab_runs(c); }

int launch_slab_stage(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, bool last) {
  if (const char *why = slab_unsupported(c)) {
    c->err = std::string("slab stage: ") + why;
    return KMY_ERR_BAD_PARAM;
  }
  if (!md0.ghosts) {
    if (const int rc = launch_fill_ghosts(c, md0)) return rc;
  }
  // constrained transport: the face-flux arrays the edge EMFs read
  if (c->prm.mhd) {
    if (const int rc = ensure_flux(c)) return rc;
    if (!md0.fc || !c->flux) {
      c->err = "slab stage: constrained transport without face arrays";
      return KMY_ERR_STATE;
    }
  }
  const MeshDesc &m = c->m;
  const bool f32 = c->esz == 4;
  CUtensorMap mc, ml;
  std::memset(&mc, 0, sizeof(mc));
  std::memset(&ml, 0, sizeof(ml));
  const int ty = slab_rows(c);
  const int ncc = c->prm.mhd ? 8 : slab::NCV;
  if (int rc = make_map(c, &mc, md0.cc, ncc, ty + 2 * slab::HH, int(c->esz))) return rc;
  if (f32) {
    if (int rc = make_map(c, &ml, md0.ener_lo, 1, ty + 2 * slab::HH, 4)) return rc;
  } else {
    ml = mc;  // no energy low words in FP64 (the kernel does not read this map)
  }
  auto fill = [&](auto &a) {
    using R = std::remove_reference_t<decltype(*a.u1)>;
    a.m = m;
    a.eos = c->eos;
    a.gm1 = R(c->eos.gm1);
    a.gam = R(c->eos.gm1 + 1.0);
    a.limiter = c->prm.limiter;
    a.u0 = static_cast<const R *>(md0.cc);
    a.u0lo = static_cast<const float *>(md0.ener_lo);
    a.ub = static_cast<const R *>(base.cc);
    a.ublo = static_cast<const float *>(base.ener_lo);
    a.u1 = static_cast<R *>(md1.cc);
    a.u1lo = static_cast<float *>(md1.ener_lo);
    a.last = last ? 1 : 0;
    a.beta = beta;
    a.clock = c->clock;
    a.rgroup = row_group(m.np[0], int(c->esz));
    a.nty = m.nx[1] / ty;
    a.nitems = m.nb * a.nty;
    a.wait_limit = 1 << 22;
    a.tx_extra = 0;
    a.fc0 = c->prm.mhd ? static_cast<const R *>(md0.fc) : nullptr;
    a.flux = c->prm.mhd ? static_cast<R *>(c->flux) : nullptr;
    if (c->fault_wait) {
      // kmy_set_fault(ctx, "stage_wait", 1): this stage's waits run out
      a.tx_extra = 16;
      a.wait_limit = 1 << 10;
    }
  };
  const int nitems = m.nb * (m.nx[1] / ty);
  const int grid = std::min(nitems, sm_count(c->device) * slab_ctas(c, ty));
  const size_t smem = size_t(slab_smem(c, ty));
  if (last) {
    k_reset_dtmin_slab<<<1, 1, 0, c->stream>>>(c->clock);
    c->launches++;
  }
  int rc;
  if (f32) {
    slab::Args<float> a{};
    fill(a);
    rc = c->prm.mhd ? slab_dispatch_mhd(c, mc, ml, a, ty, grid, smem) : slab_dispatch_f32(c, mc, ml, a, ty, grid, smem);
  } else {
    slab::Args<double> a{};
    fill(a);
    rc = slab_dispatch_f64(c, mc, ml, a, ty, grid, smem);
  }
  c->fault_wait = 0;
  md1.ghosts = rc == KMY_OK;
  return rc;
}

}  // namespace kmy

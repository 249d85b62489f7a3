// kmy_ct.cu -- the face half of a constrained-transport stage, streamed
// through each meshblock along z, and the cell pass that follows it.
//
// k_ct_emf_faces: one CTA per (meshblock, tile of TY rows by the block's 32
// columns, chunk of CT_ZC cell planes) walks the chunk's node planes.  Per
// plane it forms the edge EMFs the tile's faces need once each, into shared
// memory (CalculateEMF's arithmetic average, hydro_add_flux_tasks.cpp:387-442:
// E_x and E_y on node plane k, E_z on cell plane k), then updates the z faces
// of plane k and the x and y faces of cell plane k - 1 from them: FluxStokes
// (grid_update.hpp:80-137) and the low-storage update ApplyDuDt
// (grid.cpp:213-241; the input container's faces are left as they are),
// with the expressions of the per-face-direction kernel in the same order
// (the two compilations may contract a product into an FMA differently, an
// ulp apart).  Each face is read and written only by the
// thread that owns it, so an update in place (a stage whose output container
// is its input) is safe, and an EMF on a block face is formed by the same
// code in both blocks that share it.  The face inputs are loaded before the
// EMF barrier so the two latencies overlap; the EMF planes rotate through
// three shared buffers (a plane's faces read the buffers of planes k and
// k - 1 while the next plane is written into the third), so one barrier per
// plane suffices.  Chunks along z give the launch enough CTAs to hide the
// per-plane latency; each chunk forms its first node plane's EMFs again.
//
// k_ct_cells: the cell-centred field of md1 from its new faces (the face
// average of primconsflux.cpp:102-129), the primitives (PreparePrimitive,
// primconsflux.cpp:82-142, with the ideal-gas EOS), and on the last stage the
// CFL estimate (EstimateTimeStep, hydro_time_step.cpp:19-64) and div B in
// FP64 (FillDerived, hydro.cpp:150-190) from the same values.  When the
// z-streamed stage runs the cells, it writes the field's face ghosts instead
// of storing the primitives (that stage converts its input itself).
//
// Edges on block faces read the ghost-layer fluxes that k_flux_halo copies.
#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

namespace kmy {

namespace {

constexpr int CT_NX = 32;  // cells per block along x (one warp per row)
constexpr int CT_TY = 8;   // rows per tile
constexpr int CT_ZC = 8;   // cell planes per CTA of the face update

template <typename S, int TY>
__global__ void __launch_bounds__(CT_NX * TY)
    k_ct_emf_faces(MeshDesc m, const S *flux, const S *fb, S *f0, S *f1, double beta, const double *dt_dev,
                   const DevClock *clock) {
  constexpr int NX = CT_NX;
  __shared__ S ex[3][TY + 1][NX];      // E_x on a node plane, rows oy .. oy + TY
  __shared__ S ey[3][TY][NX + 1];      // E_y on a node plane, columns 0 .. 32
  __shared__ S ez[3][TY + 1][NX + 1];  // E_z on a cell plane
  if (clock->done) return;
  const int tid = threadIdx.x, lane = tid & 31, wr = tid >> 5;
  const int nty = m.nx[1] / TY;
  const int b = blockIdx.x / nty, oy = (blockIdx.x - b * nty) * TY;
  const int nz = m.nx[2];
  // this CTA's planes: cell planes k0 .. k1 - 1, z faces k0 .. k1 - 1 (and nz
  // on the last chunk); node plane k0's EMFs are formed again by every chunk
  const int k0 = blockIdx.y * CT_ZC, k1 = min(nz, k0 + CT_ZC);
  const bool last_tile = oy + TY == m.nx[1];
  const long long NF = (long long)m.nb * m.Pf, bo = (long long)b * m.Pf;
  // in-block face-array offsets (a block's face arrays hold fewer than 2^32)
  const unsigned sj = unsigned(m.nf[0]), sk = unsigned(m.nf[0]) * unsigned(m.nf[1]);
  auto off = [&](int k, int j, int i) {
    return unsigned(k + m.g[2]) * sk + unsigned(j + m.g[1]) * sj + unsigned(i + m.g[0]);
  };
  auto Fp = [&](int dir, int bcomp) { return flux + ((long long)dir * 8 + CMAGC0 + bcomp) * NF + bo; };
  const S *FyBx = Fp(1, 0), *FxBy = Fp(0, 1);  // E_z terms
  const S *FzBy = Fp(2, 1), *FyBz = Fp(1, 2);  // E_x terms
  const S *FxBz = Fp(0, 2), *FzBx = Fp(2, 0);  // E_y terms
  // the per-face-direction kernel's EMF expression: Fa / Fb shifted by sa / sb
  auto emf = [](const S *Fa, const S *Fb, unsigned p, unsigned sa, unsigned sb) {
    return S(1.0) * S(0.25) * (Fa[p - sa] + Fa[p] - Fb[p - sb] - Fb[p]);
  };
  const S L0 = S(m.dx[0]), L1 = S(m.dx[1]), L2 = S(m.dx[2]);
  const S ia0 = S(1.) / (S(m.area[0]) + S(1.e-36));
  const S ia1 = S(1.) / (S(m.area[1]) + S(1.e-36));
  const S ia2 = S(1.) / (S(m.area[2]) + S(1.e-36));
  const double h = *dt_dev;
  const S bt = S(beta);
  // a face's low-storage update from its base and input values.  The input
  // container's faces are not rewritten with x0 as ApplyDuDt does: the
  // low-storage scheme reads a stage's input container only in that stage
  // (in the first stage it is "base" and x0 equals its value).
  auto finish = [&](long long n, S vb, S v0, S out) {
    const S x0 = bt * vb + (S(1.0) - bt) * v0;
    f1[n] = x0 + bt * S(h) * out;
  };
  // stokes(edge, axis) of the per-face-direction kernel: sign * (L E_a - L E_b)
  auto st = [](S sign, S L, S Ea, S Eb) { return sign * (L * Ea - L * Eb); };
  // the face sums of FluxStokes
  auto xsum = [&](int qc, int q, int r, int i) {  // stokes(2, 1) + stokes(1, 2)
    S out = S(0);
    out += st(S(1.0), L2, ez[qc][r][i], ez[qc][r + 1][i]);
    out += st(S(-1.0), L1, ey[qc][r][i], ey[q][r][i]);
    return out * ia0;
  };
  auto ysum = [&](int qc, int q, int r, int i) {  // stokes(2, 0) + stokes(0, 2)
    S out = S(0);
    out += st(S(-1.0), L2, ez[qc][r][i], ez[qc][r][i + 1]);
    out += st(S(1.0), L0, ex[qc][r][i], ex[q][r][i]);
    return out * ia1;
  };
  auto zsum = [&](int q, int r, int i) {  // stokes(0, 1) + stokes(1, 0)
    S out = S(0);
    out += st(S(-1.0), L0, ex[q][r][i], ex[q][r + 1][i]);
    out += st(S(1.0), L1, ey[q][r][i], ey[q][r][i + 1]);
    return out * ia2;
  };

  for (int kk = k0; kk <= k1; kk++) {
    const int q = kk % 3, qc = (kk + 2) % 3;  // buffers of planes kk and kk - 1
    const bool zf = kk < k1 || kk == nz;      // this chunk updates z face kk
    const bool xy = kk > k0;                  // ... and the x and y faces of cell plane kk - 1
    // the owned faces' inputs, loaded ahead so their latency overlaps the EMFs'
    const long long nz_ = 2 * NF + bo + off(kk, oy + wr, lane);
    const long long nx_ = bo + off(kk - 1, oy + wr, lane), ny_ = NF + nx_;
    S zb = S(0), z0 = S(0), xb = S(0), x0 = S(0), yb = S(0), y0 = S(0);
    if (zf) {
      zb = fb[nz_];
      z0 = f0[nz_];
    }
    if (xy) {
      xb = fb[nx_];
      x0 = f0[nx_];
      yb = fb[ny_];
      y0 = f0[ny_];
    }
    // ---- EMFs of node plane kk (E_x, E_y) and cell plane kk (E_z) ----
    {
      auto put_ex = [&](int r, int i) { ex[q][r][i] = emf(FzBy, FyBz, off(kk, oy + r, i), sj, sk); };
      auto put_ey = [&](int r, int i) { ey[q][r][i] = emf(FxBz, FzBx, off(kk, oy + r, i), sk, 1u); };
      auto put_ez = [&](int r, int i) { ez[q][r][i] = emf(FyBx, FxBy, off(kk, oy + r, i), 1u, sj); };
      put_ex(wr, lane);
      put_ey(wr, lane);
      if (tid < NX) put_ex(TY, tid);
      if (tid < TY) put_ey(tid, NX);
      if (kk < k1) {
        put_ez(wr, lane);
        if (tid < NX) put_ez(TY, tid);
        if (tid < TY + 1) put_ez(tid, NX);
      }
    }
    __syncthreads();
    if (zf) finish(nz_, zb, z0, zsum(q, wr, lane));
    if (xy) {
      finish(nx_, xb, x0, xsum(qc, q, wr, lane));
      finish(ny_, yb, y0, ysum(qc, q, wr, lane));
      if (tid < TY) {  // x faces at i = 32
        const long long n = bo + off(kk - 1, oy + tid, NX);
        finish(n, fb[n], f0[n], xsum(qc, q, tid, NX));
      }
      if (last_tile && tid < NX) {  // y faces at j = ny
        const long long n = NF + bo + off(kk - 1, oy + TY, tid);
        finish(n, fb[n], f0[n], ysum(qc, q, TY, tid));
      }
    }
  }
}

// The face ghosts of a cell's new field components, for a z-streamed stage
// that stages the next stage's input with its ghost zones: an interior cell
// within g of a block face fills the ghosts that Parthenon's boundary
// exchange would fill from it (the high ghosts of the block below along an
// axis, the low ghosts of the block above, wrapped across a periodic
// boundary; at an outflow boundary its own block's ghosts; at a reflecting
// one the mirror with the normal component negated), the rule of the
// z-streamed stage's epilogue.  pc: the cell's padded coordinates.
template <typename S>
__device__ void push_field_ghosts(const MeshDesc &m, S *cc, long long NP, int b, const int pc[3],
                                  const S (&B)[3]) {
  const int lb[3] = {b % m.nbx[0], (b / m.nbx[0]) % m.nbx[1], b / (m.nbx[0] * m.nbx[1])};
  auto store = [&](long long idx, int flip) {
#pragma unroll
    for (int q = 0; q < 3; q++) cc[(CMAGC0 + q) * NP + idx] = q == flip ? -B[q] : B[q];
  };
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int n = m.nx[d], g = m.g[d], nbd = m.nbx[d];
    const int l = pc[d] - g;
    if (l >= g && l < n - g) continue;
    const long long stride = d == 0 ? 1 : d == 1 ? m.nbx[0] : (long long)m.nbx[0] * m.nbx[1];
    // element offset of pc with coordinate d replaced by p, in block tb
    auto at = [&](long long tb, int p) {
      int q[3] = {pc[0], pc[1], pc[2]};
      q[d] = p;
      return tb * m.P + ((long long)q[2] * m.np[1] + q[1]) * m.np[0] + q[0];
    };
    if (l < g) {
      if (lb[d] > 0 || m.bc[d][0] == BC_PERIODIC) {
        store(at(b + (lb[d] > 0 ? -stride : (long long)(nbd - 1) * stride), n + g + l), -1);
      } else if (m.bc[d][0] == BC_OUTFLOW) {
        if (l == 0)
          for (int p = 0; p < g; p++) store(at(b, p), -1);
      } else {
        store(at(b, g - 1 - l), d);
      }
    }
    if (l >= n - g) {
      if (lb[d] < nbd - 1 || m.bc[d][1] == BC_PERIODIC) {
        store(at(b + (lb[d] < nbd - 1 ? stride : -(long long)(nbd - 1) * stride), l - n + g), -1);
      } else if (m.bc[d][1] == BC_OUTFLOW) {
        if (l == n - 1)
          for (int p = 0; p < g; p++) store(at(b, n + g + p), -1);
      } else {
        store(at(b, g + 2 * n - 1 - l), d);
      }
    }
  }
}

// One thread per column of a CTA of 8 rows of one block; the CTA walks a
// chunk of CT_ZC planes (on the last stage one atomic per CTA collects the
// CFL minimum, so fewer, longer CTAs keep that atomic off the critical path).
template <typename S, bool LAST>
__global__ void __launch_bounds__(CT_NX * CT_TY)
    k_ct_cells(MeshDesc m, EosParams eos, S *cc, const float *lo, const S *fc, S *prim, double *divb,
               DevClock *clock, int push) {
  // push: the z-streamed stage runs the cells; it stages the next input with
  // its ghost zones (so the field's face ghosts are written here) and converts
  // it itself (so the primitives are not stored)
  __shared__ double wmin[CT_TY];
  const int tid = threadIdx.x, lane = tid & 31, wr = tid >> 5;
  const int nty = m.nx[1] / CT_TY;
  const int b = blockIdx.x / nty, oy = (blockIdx.x - b * nty) * CT_TY;
  const int k0 = blockIdx.y * CT_ZC, k1 = min(m.nx[2], k0 + CT_ZC);
  const int i = lane + m.g[0], j = oy + wr + m.g[1];
  const long long NP = (long long)m.nb * m.P, NF = (long long)m.nb * m.Pf, bo = (long long)b * m.Pf;
  auto fo = [&](int kk, int jj, int ii) { return bo + ((long long)kk * m.nf[1] + jj) * m.nf[0] + ii; };
  const S vol = S(m.vol);
  const S a0 = S(m.area[0]), a1 = S(m.area[1]), a2 = S(m.area[2]);
  double dtl = INFINITY;
  for (int k = k0; k < k1; k++) {
    const int kp = k + m.g[2];
    const long long n = (long long)b * m.P + ((long long)kp * m.np[1] + j) * m.np[0] + i;
    const long long f000 = fo(kp, j, i), fx1 = fo(kp, j, i + 1), fy1 = fo(kp, j + 1, i), fz1 = fo(kp + 1, j, i);
    // the face average (primconsflux.cpp:102-129)
    S B[3];
    B[0] = S(0.5) * S(m.dx[0]) * (a0 * fc[fx1] + a0 * fc[f000]) / vol;
    B[1] = S(0.5) * S(m.dx[1]) * (a1 * fc[NF + fy1] + a1 * fc[NF + f000]) / vol;
    B[2] = S(0.5) * S(m.dx[2]) * (a2 * fc[2 * NF + fz1] + a2 * fc[2 * NF + f000]) / vol;
#pragma unroll
    for (int d = 0; d < 3; d++) cc[(CMAGC0 + d) * NP + n] = B[d];
    if (push) {
      const int pc[3] = {i, j, kp};
      push_field_ghosts(m, cc, NP, b, pc, B);
    }
    if (push && !LAST) continue;  // nothing else to do for this cell
    double ener = double(cc[CENER * NP + n]);
    if constexpr (sizeof(S) == 4) {
      if (lo) ener += double(lo[n]);
    }
    S V[10];
    Cons2PrimEos<true, S>(eos, cc[n], cc[CMOM0 * NP + n], cc[CMOM1 * NP + n], cc[CMOM2 * NP + n], ener, B, V);
    if (!push) {
      prim[PVEL0 * NP + n] = V[RVEL0];
      prim[PVEL1 * NP + n] = V[RVEL1];
      prim[PVEL2 * NP + n] = V[RVEL2];
      prim[PPRES * NP + n] = V[RPRES];
      prim[PBMOD * NP + n] = V[RBMOD];
      prim[PEINT * NP + n] = V[REINT];
      prim[PTEMP * NP + n] = kmax(S(0), V[REINT] / S(eos.cv));
    }
    if constexpr (LAST) {
      // div B in FP64 (hydro.cpp:150-190)
      double d = 0.;
      d += m.area[0] * double(fc[fx1]) - m.area[0] * double(fc[f000]);
      d += m.area[1] * double(fc[NF + fy1]) - m.area[1] * double(fc[NF + f000]);
      d += m.area[2] * double(fc[2 * NF + fz1]) - m.area[2] * double(fc[2 * NF + f000]);
      divb[n] = d / m.vol;
      // CFL estimate (hydro_time_step.cpp:19-64); a NaN propagates
#pragma unroll
      for (int dir = 0; dir < 3; dir++) {
        const S cf = FastSpeed<true>(dir, V);
        const double x = double(S(m.dx[dir]) / (fabs(V[RVEL0 + dir]) + cf));
        dtl = (x < dtl || x != x) ? x : dtl;
      }
    }
  }
  if constexpr (LAST) {
    for (int o = 16; o > 0; o >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, o));
    if (lane == 0) wmin[wr] = dtl;
    __syncthreads();
    if (tid == 0) {
      double v = wmin[0];
      for (int w = 1; w < CT_TY; w++) v = fmin(v, wmin[w]);
      if (!(v >= 0.0)) v = 0.0;  // NaN or negative: 0, which the dt controller flags
      atomicMin(&clock->dtmin_bits, (unsigned long long)__double_as_longlong(v));
    }
  }
}

__global__ void k_ct_reset_dtmin(DevClock *clock) { clock->dtmin_bits = 0x7FF0000000000000ull; }

template <typename S>
int ct_launch(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, bool fold_last) {
  const MeshDesc &m = c->m;
  const unsigned tiles = unsigned(m.nb) * unsigned(m.nx[1] / CT_TY);
  const dim3 fgrid(tiles, unsigned((m.nx[2] + CT_ZC - 1) / CT_ZC));
  k_ct_emf_faces<S, CT_TY><<<fgrid, CT_NX * CT_TY, 0, c->stream>>>(
      m, (const S *)c->flux, (const S *)base.fc, (S *)md0.fc, (S *)md1.fc, beta, &c->clock->dt, c->clock);
  c->launches++;
  const dim3 grid(tiles, unsigned((m.nx[2] + CT_ZC - 1) / CT_ZC));
  // the field's face ghosts, for the z-streamed stage that stages md1 next
  const int push = ct_cells_on_slab(c) ? 1 : 0;
  const float *lo = c->esz == 4 ? static_cast<const float *>(md1.ener_lo) : nullptr;
  if (fold_last) {
    k_ct_reset_dtmin<<<1, 1, 0, c->stream>>>(c->clock);
    k_ct_cells<S, true><<<grid, CT_NX * CT_TY, 0, c->stream>>>(m, c->eos, (S *)md1.cc, lo, (const S *)md1.fc,
                                                               (S *)c->prim, c->divb, c->clock, push);
    c->launches += 2;
  } else {
    k_ct_cells<S, false><<<grid, CT_NX * CT_TY, 0, c->stream>>>(m, c->eos, (S *)md1.cc, lo, (const S *)md1.fc,
                                                                (S *)c->prim, c->divb, c->clock, push);
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "ct stream");
}

}  // namespace

const char *ct_stream_unsupported(const kmy_ctx *c) {
  const MeshDesc &m = c->m;
  if (!c->prm.mhd) return "no constrained transport";
  if (c->prm.ct_update == 2) return "the deck asks for the per-face-direction update";
  if (m.ndim != 3) return "the streamed face update is 3D";
  if (c->amr.on || m.blev) return "adaptive meshes run the per-face-direction update";
  if (m.nx[0] != CT_NX) return "the streamed face update needs 32 cells per block along x";
  if (m.nx[1] % CT_TY) return "the block height is not a multiple of 8";
  if (m.Pf * 3 >= (1ll << 32)) return "face arrays too large for 32-bit in-block offsets";
  return nullptr;
}

int launch_ct_stream(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, bool fold_last) {
  if (const char *why = ct_stream_unsupported(c)) {
    c->err = std::string("ct stream: ") + why;
    return KMY_ERR_BAD_PARAM;
  }
  return c->esz == 8 ? ct_launch<double>(c, base, md0, md1, beta, fold_last)
                     : ct_launch<float>(c, base, md0, md1, beta, fold_last);
}

}  // namespace kmy

// kmy_tasks.cu -- per-task kernels at the reference's task granularity, on the
// full ghost-padded MeshData layout: face fluxes, CT EMFs, flux divergence and
// Stokes face update, the low-storage RK update, cons->prim + EOS, boundary
// exchange on a single-level mesh, the CFL reduction, div B, initialisation
// kernels and the device-side dt controller.
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

namespace kmy {

constexpr int kThreads = 256;

__device__ __forceinline__ long long cidx(const MeshDesc &m, int k, int j, int i) {
  return ((long long)k * m.np[1] + j) * m.np[0] + i;
}
__device__ __forceinline__ long long fidx(const MeshDesc &m, int k, int j, int i) {
  return ((long long)k * m.nf[1] + j) * m.nf[0] + i;
}
__device__ __forceinline__ int block_loc(const MeshDesc &m, int b, int d) {
  if (d == 0) return b % m.nbx[0];
  if (d == 1) return (b / m.nbx[0]) % m.nbx[1];
  return b / (m.nbx[0] * m.nbx[1]);
}

// Energy of cell n as double (FP32 storage keeps E as hi + lo floats).
template <typename S>
__device__ __forceinline__ double load_ener(const S *cc, const float *lo, long long stride, long long n) {
  double e = double(cc[CENER * stride + n]);
  if constexpr (sizeof(S) == 4) {
    if (lo) e += double(lo[n]);
  }
  return e;
}
template <typename S>
__device__ __forceinline__ void store_ener(S *cc, float *lo, long long stride, long long n, double e) {
  if constexpr (sizeof(S) == 4) {
    const float hi = float(e);
    cc[CENER * stride + n] = hi;
    if (lo) lo[n] = float(e - double(hi));
  } else {
    cc[CENER * stride + n] = e;
  }
}

// Flat thread index t (< per * nblocks) -> block b and cell (i, j, k) of an
// n0 x n1 x (per / (n0 n1)) range.  Unsigned 32-bit division whenever the
// numbers fit, which every launch of a mesh below 2^32 cells does; 64-bit
// integer division is a long software sequence on the GPU.
__device__ __forceinline__ void unflatten(long long t, long long per, int n0, int n1, int &b, int &i, int &j,
                                          int &k) {
  if (t < (1LL << 32) && per < (1LL << 32)) {
    const unsigned u = unsigned(t), p = unsigned(per);
    const unsigned bb = u / p, r = u - bb * p;
    const unsigned q = r / unsigned(n0);
    b = int(bb);
    i = int(r - q * unsigned(n0));
    j = int(q % unsigned(n1));
    k = int(q / unsigned(n1));
  } else {
    b = int(t / per);
    long long r = t - (long long)b * per;
    i = int(r % n0);
    r /= n0;
    j = int(r % n1);
    k = int(r / n1);
  }
}

static unsigned nblk(long long n) { return unsigned((n + kThreads - 1) / kThreads); }

// ---------------------------------------------------------------------------
// Boundary exchange on a single level (Parthenon AddBoundaryExchangeTasks with
// periodic / outflow / reflect physical boundaries).  Every ghost cell copies
// the interior cell it maps to; reflect flips normal vector components.
__device__ __forceinline__ int map_index(int G, int N, int bc, bool &flip) {
  if (G >= 0 && G < N) return G;
  if (bc == BC_PERIODIC) return ((G % N) + N) % N;
  if (bc == BC_OUTFLOW) return G < 0 ? 0 : N - 1;
  flip = !flip;
  return G < 0 ? -G - 1 : 2 * N - G - 1;
}

template <typename S>
__global__ void k_fill_ghost_cells(MeshDesc m, S *cc, float *lo, S *prim, int ncc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)m.nb * m.P) return;
  int b, i, j, k;
  unflatten(t, m.P, m.np[0], m.np[1], b, i, j, k);
  const int loc[3] = {i, j, k};
  bool interior = true;
  for (int d = 0; d < 3; d++)
    if (loc[d] < m.g[d] || loc[d] >= m.g[d] + m.nx[d]) interior = false;
  if (interior) return;
  int src[3], sb = 0, mult = 1;
  bool flip[3] = {false, false, false};
  for (int d = 0; d < 3; d++) {
    const int G = block_loc(m, b, d) * m.nx[d] + (loc[d] - m.g[d]);
    const int N = m.mesh_nx[d];
    const int M = map_index(G, N, m.bc[d][G < 0 ? 0 : 1], flip[d]);
    sb += (M / m.nx[d]) * mult;
    mult *= m.nbx[d];
    src[d] = M % m.nx[d] + m.g[d];
  }
  const long long NP = (long long)m.nb * m.P;
  const long long dst = (long long)b * m.P + cidx(m, k, j, i);
  const long long s = (long long)sb * m.P + cidx(m, src[2], src[1], src[0]);
  for (int v = 0; v < ncc; v++) {
    S val = cc[v * NP + s];
    if (v >= CMOM0 && v <= CMOM2 && flip[v - CMOM0]) val = -val;
    if (v >= CMAGC0 && flip[v - CMAGC0]) val = -val;
    cc[v * NP + dst] = val;
  }
  if constexpr (sizeof(S) == 4) {
    if (lo) lo[dst] = lo[s];
  }
  for (int v = 0; v < NPRIM; v++) {
    S val = prim[v * NP + s];
    if (v <= PVEL2 && flip[v]) val = -val;
    prim[v * NP + dst] = val;
  }
}

// Face field ghosts: a ghost face takes the value of the interior face of the
// block that owns its global position (shared block faces are left alone).
template <typename S>
__global__ void k_fill_ghost_faces(MeshDesc m, S *fc, int e) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)m.nb * m.Pf) return;
  int b, i, j, k;
  unflatten(t, m.Pf, m.nf[0], m.nf[1], b, i, j, k);
  const int loc[3] = {i, j, k};
  for (int d = 0; d < 3; d++)
    if (loc[d] >= m.np[d] + (d == e ? 1 : 0)) return;  // outside this element's extent
  bool interior = true;
  for (int d = 0; d < 3; d++) {
    const int hi = m.g[d] + m.nx[d] - 1 + (d == e ? 1 : 0);
    if (loc[d] < m.g[d] || loc[d] > hi) interior = false;
  }
  if (interior) return;
  int src[3], sb = 0, mult = 1;
  for (int d = 0; d < 3; d++) {
    const int G = block_loc(m, b, d) * m.nx[d] + (loc[d] - m.g[d]);
    const int N = m.mesh_nx[d];
    int M;
    if (d == e) {
      if (G >= 0 && G <= N) M = G;
      else if (m.bc[d][G < 0 ? 0 : 1] == BC_PERIODIC) M = ((G % N) + N) % N;
      else M = G < 0 ? 0 : N;
    } else {
      bool f = false;
      M = map_index(G, N, m.bc[d][G < 0 ? 0 : 1], f);
    }
    int owner = M / m.nx[d];
    if (owner >= m.nbx[d]) owner = m.nbx[d] - 1;
    sb += owner * mult;
    mult *= m.nbx[d];
    src[d] = M - owner * m.nx[d] + m.g[d];
  }
  const long long NF = (long long)m.nb * m.Pf;
  fc[e * NF + (long long)b * m.Pf + fidx(m, k, j, i)] =
      fc[e * NF + (long long)sb * m.Pf + fidx(m, src[2], src[1], src[0])];
}

int launch_fill_ghosts(kmy_ctx *c, Container &ct) {
  if (c->amr.on) return launch_amr_fill_ghosts(c, ct);
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nb * m.P;
  if (c->esz == 8)
    k_fill_ghost_cells<double><<<nblk(n), kThreads, 0, c->stream>>>(
        m, (double *)ct.cc, nullptr, (double *)c->prim, c->ncc);
  else
    k_fill_ghost_cells<float><<<nblk(n), kThreads, 0, c->stream>>>(
        m, (float *)ct.cc, (float *)ct.ener_lo, (float *)c->prim, c->ncc);
  c->launches++;
  if (c->prm.mhd) {
    const long long nf = (long long)m.nb * m.Pf;
    for (int e = 0; e < m.ndim; e++) {
      if (c->esz == 8)
        k_fill_ghost_faces<double><<<nblk(nf), kThreads, 0, c->stream>>>(m, (double *)ct.fc, e);
      else
        k_fill_ghost_faces<float><<<nblk(nf), kThreads, 0, c->stream>>>(m, (float *)ct.fc, e);
      c->launches++;
    }
  }
  const int rc = cuda_check(c, cudaGetLastError(), "fill_ghosts");
  ct.ghosts = rc == KMY_OK;
  return rc;
}

// ---------------------------------------------------------------------------
// CalculateFluxesNested (hydro_add_flux_tasks.cpp:36-264): one thread per face
// of direction DIR.  Reconstruction of every primitive at the two cells that
// share the face, CT face-field override, then the Riemann flux.
template <typename S, int RECON, int RIEMANN, bool MHD, int DIR>
__global__ void k_face_flux(MeshDesc m, int limiter, const S *cc, const S *prim, const S *fc,
                            S *flux, int lo0, int lo1, int lo2, int n0, int n1, int n2) {
  constexpr int NR = MHD ? 10 : 7;
  constexpr int NC = MHD ? 8 : 5;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)n0 * n1 * n2;
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, n0, n1, b, i, j, k);
  i += lo0;
  j += lo1;
  k += lo2;
  const long long NP = (long long)m.nb * m.P;
  const long long base = (long long)b * m.P + cidx(m, k, j, i);
  const long long st = DIR == 0 ? 1 : DIR == 1 ? m.np[0] : (long long)m.np[0] * m.np[1];
  constexpr int W = ReconWidth<RECON>::value;
  S vL[NR], vR[NR];
#pragma unroll
  for (int rv = 0; rv < NR; rv++) {
    const S *src;
    if (rv == RDENS) src = cc;
    else if (rv <= RVEL2) src = prim + (PVEL0 + rv - RVEL0) * NP;
    else if (rv == RPRES) src = prim + PPRES * NP;
    else if (rv == RBMOD) src = prim + PBMOD * NP;
    else if (rv == REINT) src = prim + PEINT * NP;
    else src = cc + (CMAGC0 + rv - RMAGC0) * NP;
    // cells f-1-W .. f+W along DIR (f = this face's high cell)
    S line[2 * W + 2];
#pragma unroll
    for (int o = 0; o < 2 * W + 2; o++) line[o] = src[base + (o - 1 - W) * st];
    S sl[5], sr[5];
#pragma unroll
    for (int o = 0; o < 5; o++) {
      const int ol = o - 2 + W;      // index of (f-1) + (o-2) in line
      const int orr = o - 2 + W + 1; // index of f + (o-2) in line
      sl[o] = (ol >= 0 && ol < 2 * W + 2) ? line[ol] : S(0);
      sr[o] = (orr >= 0 && orr < 2 * W + 2) ? line[orr] : S(0);
    }
    vL[rv] = ReconstructPlus<RECON, S>(limiter, sl);
    vR[rv] = ReconstructMinus<RECON, S>(limiter, sr);
  }
  if constexpr (MHD) {
    const long long NF = (long long)m.nb * m.Pf;
    const S bn = fc[DIR * NF + (long long)b * m.Pf + fidx(m, k, j, i)];
    vL[RMAGC0 + DIR] = bn;
    vR[RMAGC0 + DIR] = bn;
  }
  S F[NC];
  RiemannFlux<RIEMANN, MHD, DIR, S>(vL, vR, F);
  const long long NF = (long long)m.nb * m.Pf;
  const long long fo = (long long)b * m.Pf + fidx(m, k, j, i);
#pragma unroll
  for (int v = 0; v < NC; v++) flux[((long long)DIR * NC + v) * NF + fo] = F[v];
}

template <typename S, int RECON, int RIEMANN, bool MHD>
static void face_flux_dir(kmy_ctx *c, int dir, const S *cc, const S *prim, const S *fc, S *flux) {
  const MeshDesc &m = c->m;
  int lo[3], n[3];
  for (int d = 0; d < 3; d++) {
    int s = m.g[d], e = m.g[d] + m.nx[d] - 1;
    if (MHD && d < m.ndim && m.ndim > 1) {  // widened bounds for the edge EMFs (:59-70)
      s -= 1;
      e += 1;
    }
    if (d == dir) e += 1;  // faces s .. e+1
    lo[d] = s;
    n[d] = e - s + 1;
  }
  const long long tot = (long long)n[0] * n[1] * n[2] * m.nb;
  const int lim = c->prm.limiter;
  if (dir == 0)
    k_face_flux<S, RECON, RIEMANN, MHD, 0><<<nblk(tot), kThreads, 0, c->stream>>>(
        m, lim, cc, prim, fc, flux, lo[0], lo[1], lo[2], n[0], n[1], n[2]);
  else if (dir == 1)
    k_face_flux<S, RECON, RIEMANN, MHD, 1><<<nblk(tot), kThreads, 0, c->stream>>>(
        m, lim, cc, prim, fc, flux, lo[0], lo[1], lo[2], n[0], n[1], n[2]);
  else
    k_face_flux<S, RECON, RIEMANN, MHD, 2><<<nblk(tot), kThreads, 0, c->stream>>>(
        m, lim, cc, prim, fc, flux, lo[0], lo[1], lo[2], n[0], n[1], n[2]);
  c->launches++;
}

// Face flux storage, [dir][ncc][nb * Pf], allocated on first use.
int ensure_flux(kmy_ctx *c) {
  if (c->flux) return KMY_OK;
  return dalloc(c, &c->flux, c->esz * 3 * c->ncc * size_t(c->m.nb) * c->m.Pf);
}

template <typename S>
static int compute_fluxes_t(kmy_ctx *c, Container &md0) {
  const MeshDesc &m = c->m;
  if (const int rc = ensure_flux(c)) return rc;
  const S *cc = (const S *)md0.cc, *prim = (const S *)c->prim, *fc = (const S *)md0.fc;
  S *flux = (S *)c->flux;
  const int rec = c->prm.recon, rie = c->prm.riemann;
  const bool mhd = c->prm.mhd;
  for (int dir = 0; dir < m.ndim; dir++) {
#define KMY_FF(R_, RI_, M_) face_flux_dir<S, R_, RI_, M_>(c, dir, cc, prim, fc, flux)
#define KMY_FF_R(R_)                                       \
  if (rie == HLL) {                                        \
    if (mhd) KMY_FF(R_, HLL, true); else KMY_FF(R_, HLL, false);   \
  } else {                                                 \
    if (mhd) KMY_FF(R_, HLLC, true); else KMY_FF(R_, HLLC, false); \
  }
    if (rec == FOG) { KMY_FF_R(FOG) }
    else if (rec == PLM) { KMY_FF_R(PLM) }
    else if (rec == PPM) { KMY_FF_R(PPM) }
    else { KMY_FF_R(WENOZ) }
#undef KMY_FF_R
#undef KMY_FF
  }
  return cuda_check(c, cudaGetLastError(), "compute_fluxes");
}

int launch_compute_fluxes(kmy_ctx *c, Container &md0) {
  return c->esz == 8 ? compute_fluxes_t<double>(c, md0) : compute_fluxes_t<float>(c, md0);
}

// ---------------------------------------------------------------------------
// Ghost-layer transverse field fluxes for the edge EMFs.  The fused stage
// computes face fluxes on interior faces only; the EMF of an edge on a block
// face also reads F_a[B_t] one cell row outside the block across t.  On a
// single-level mesh with periodic or outflow boundaries that row is the
// interior row of the block owning it (or the boundary row itself, for
// outflow), as the boundary exchange would have filled the cells the flux
// came from, so the flux is copied from there.  One thread per ghost-layer
// face: face direction a, transverse axis t, side, the a-face index and the
// remaining axis c.
// One launch covers every (face direction a, transverse axis t) pair of the
// mesh: blockIdx.y indexes the pairs ((a, t) in pairs[], na and nc per pair).
struct FluxHaloPairs {
  int n;
  int a[6], t[6], na[6], nc[6];
};

template <typename S>
__global__ void k_flux_halo(MeshDesc m, S *flux, FluxHaloPairs pairs) {
  const int pi = blockIdx.y;
  const int a = pairs.a[pi], t = pairs.t[pi], na = pairs.na[pi], nc = pairs.nc[pi];
  const int cax = 3 - a - t;
  const long long tt = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = 2LL * na * nc;
  if (tt >= per * m.nb) return;
  const int b = int(tt / per);
  int r = int(tt - (long long)b * per);
  const int side = r / (na * nc);
  r -= side * na * nc;
  const int ia = r % na, ic = r / na;
  int lb[3] = {block_loc(m, b, 0), block_loc(m, b, 1), block_loc(m, b, 2)};
  // destination: ghost row -1 or nx_t across t
  int L[3];
  L[a] = ia;
  L[cax] = ic;
  L[t] = side ? m.nx[t] : -1;
  // source: the interior row that ghost row maps to
  bool flip = false;
  const int G = lb[t] * m.nx[t] + L[t];
  const int M = map_index(G, m.mesh_nx[t], m.bc[t][side], flip);
  const int ob = M / m.nx[t];
  int Ls[3] = {L[0], L[1], L[2]};
  Ls[t] = M - ob * m.nx[t];
  int sb[3] = {lb[0], lb[1], lb[2]};
  sb[t] = ob;
  const int bs = sb[0] + m.nbx[0] * (sb[1] + m.nbx[1] * sb[2]);
  const long long NF = (long long)m.nb * m.Pf;
  S *F = flux + ((long long)a * 8 + CMAGC0 + t) * NF;
  F[(long long)b * m.Pf + fidx(m, L[2] + m.g[2], L[1] + m.g[1], L[0] + m.g[0])] =
      F[(long long)bs * m.Pf + fidx(m, Ls[2] + m.g[2], Ls[1] + m.g[1], Ls[0] + m.g[0])];
}

int launch_flux_halo(kmy_ctx *c) {
  const MeshDesc &m = c->m;
  FluxHaloPairs p{};
  long long most = 0;
  for (int a = 0; a < m.ndim; a++)
    for (int t = 0; t < m.ndim; t++) {
      if (t == a) continue;
      p.a[p.n] = a;
      p.t[p.n] = t;
      p.na[p.n] = m.nx[a] + 1;
      p.nc[p.n] = m.nx[3 - a - t];
      most = std::max(most, 2LL * p.na[p.n] * p.nc[p.n] * m.nb);
      p.n++;
    }
  if (!p.n) return KMY_OK;
  const dim3 grid(nblk(most), unsigned(p.n));
  if (c->esz == 8)
    k_flux_halo<double><<<grid, kThreads, 0, c->stream>>>(m, (double *)c->flux, p);
  else
    k_flux_halo<float><<<grid, kThreads, 0, c->stream>>>(m, (float *)c->flux, p);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "flux_halo");
}

// ---------------------------------------------------------------------------
// CalculateEMF (hydro_add_flux_tasks.cpp:387-442), arithmetic averaging.  Each
// edge family over its own interior edge range.
template <typename S>
__global__ void k_edge_emf(MeshDesc m, const S *flux, S *emf, int e, int n0, int n1, int n2) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)n0 * n1 * n2;
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, n0, n1, b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf;
  const long long bo = (long long)b * m.Pf;
  auto F = [&](int dir, int bcomp, int kk, int jj, int ii) {
    return flux[((long long)dir * 8 + CMAGC0 + bcomp) * NF + bo + fidx(m, kk, jj, ii)];
  };
  S val;
  if (e == 2)
    val = S(1.0) * S(0.25) * (F(1, 0, k, j, i - 1) + F(1, 0, k, j, i) - F(0, 1, k, j - 1, i) - F(0, 1, k, j, i));
  else if (e == 0)
    val = S(1.0) * S(0.25) * (F(2, 1, k, j - 1, i) + F(2, 1, k, j, i) - F(1, 2, k - 1, j, i) - F(1, 2, k, j, i));
  else
    val = S(1.0) * S(0.25) * (F(0, 2, k - 1, j, i) + F(0, 2, k, j, i) - F(2, 0, k, j, i - 1) - F(2, 0, k, j, i));
  emf[e * NF + bo + fidx(m, k, j, i)] = val;
}

int launch_compute_emf(kmy_ctx *c, Container &md0) {
  const MeshDesc &m = c->m;
  if (!c->prm.mhd || m.ndim < 2) return KMY_OK;
  for (int e = (m.ndim > 2 ? 0 : 2); e < 3; e++) {
    // node-like (+1) in the two directions normal to the edge
    int n[3];
    for (int d = 0; d < 3; d++) n[d] = m.nx[d] + ((d != e && d < m.ndim) ? 1 : 0);
    const long long tot = (long long)n[0] * n[1] * n[2] * m.nb;
    if (c->esz == 8)
      k_edge_emf<double><<<nblk(tot), kThreads, 0, c->stream>>>(m, (const double *)c->flux,
                                                                  (double *)md0.emf, e, n[0], n[1], n[2]);
    else
      k_edge_emf<float><<<nblk(tot), kThreads, 0, c->stream>>>(m, (const float *)c->flux,
                                                                 (float *)md0.emf, e, n[0], n[1], n[2]);
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "compute_emf");
}

// ---------------------------------------------------------------------------
// FluxDivergence (grid_update.hpp:15-57)
template <typename S>
__global__ void k_flux_divergence(MeshDesc m, const S *flux, S *du, int ncc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf, NP = (long long)m.nb * m.P;
  const long long bo = (long long)b * m.Pf;
  for (int v = 0; v < ncc; v++) {
    S d = S(0);
    for (int dir = 0; dir < m.ndim; dir++) {
      const int kp = k + (dir == 2), jp = j + (dir == 1), ip = i + (dir == 0);
      const S A = S(blk_area(m, b, dir));
      const S *F = flux + ((long long)dir * ncc + v) * NF + bo;
      d -= (A * F[fidx(m, kp, jp, ip)] - A * F[fidx(m, k, j, i)]);
    }
    du[v * NP + (long long)b * m.P + cidx(m, k, j, i)] = d / S(blk_vol(m, b));
  }
}

// FluxStokes (grid_update.hpp:80-137) for face `face` with its one or two edges.
template <typename S>
__global__ void k_flux_stokes(MeshDesc m, const S *emf, S *dufc, int face, int ne, int e0, int e1) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int n0 = m.nx[0] + (face == 0), n1 = m.nx[1] + (face == 1), n2 = m.nx[2] + (face == 2);
  const long long per = (long long)n0 * n1 * n2;
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, n0, n1, b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf, bo = (long long)b * m.Pf;
  S out = S(0);
  const int edges[2] = {e0, e1};
  for (int q = 0; q < ne; q++) {
    const int edge = edges[q];
    int axis;  // AxisFromFaceEdge, i=0 j=1 k=2
    if (face == 0) axis = edge == 2 ? 1 : 2;
    else if (face == 1) axis = edge == 2 ? 0 : 2;
    else axis = edge == 0 ? 1 : 0;
    int ijk[3] = {i, j, k};
    ijk[axis] += 1;
    const S sign = ((axis + 1) % 3 == edge) ? S(1.0) : S(-1.0);
    const S L = S(blk_dx(m, b, edge));
    const S *E = emf + edge * NF + bo;
    out += sign * (L * E[fidx(m, k, j, i)] - L * E[fidx(m, ijk[2], ijk[1], ijk[0])]);
  }
  out *= S(1.) / (S(blk_area(m, b, face)) + S(1.e-36));
  dufc[face * NF + bo + fidx(m, k, j, i)] = out;
}

int launch_flux_divergence(kmy_ctx *c, Container &md0, Container &dudt) {
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  if (c->esz == 8)
    k_flux_divergence<double><<<nblk(n), kThreads, 0, c->stream>>>(m, (const double *)c->flux,
                                                                     (double *)dudt.cc, c->ncc);
  else
    k_flux_divergence<float><<<nblk(n), kThreads, 0, c->stream>>>(m, (const float *)c->flux,
                                                                    (float *)dudt.cc, c->ncc);
  c->launches++;
  if (c->prm.mhd && m.ndim > 1) return launch_flux_stokes(c, md0, dudt);
  return cuda_check(c, cudaGetLastError(), "flux_divergence");
}

// FluxStokes for every active face direction: dU/dt of the face field from
// md0's edge EMFs.
int launch_flux_stokes(kmy_ctx *c, Container &md0, Container &dudt) {
  const MeshDesc &m = c->m;
  struct FE { int face, ne, e0, e1; };
  const FE l3[3] = {{0, 2, 2, 1}, {1, 2, 2, 0}, {2, 2, 0, 1}};
  const FE l2[2] = {{0, 1, 2, 0}, {1, 1, 2, 0}};
  const FE *l = m.ndim > 2 ? l3 : l2;
  for (int f = 0; f < m.ndim; f++) {
    const FE fe = l[f];
    const long long nfc = (long long)(m.nx[0] + (fe.face == 0)) * (m.nx[1] + (fe.face == 1)) *
                          (m.nx[2] + (fe.face == 2)) * m.nb;
    if (c->esz == 8)
      k_flux_stokes<double><<<nblk(nfc), kThreads, 0, c->stream>>>(
          m, (const double *)md0.emf, (double *)dudt.fc, fe.face, fe.ne, fe.e0, fe.e1);
    else
      k_flux_stokes<float><<<nblk(nfc), kThreads, 0, c->stream>>>(
          m, (const float *)md0.emf, (float *)dudt.fc, fe.face, fe.ne, fe.e0, fe.e1);
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "flux_divergence");
}

// ---------------------------------------------------------------------------
// ApplyDuDt_impl (grid.cpp:213-241): u0 <- beta*base + (1-beta)*u0 ; u1 <- u0 + beta*dt*du
template <typename S>
__global__ void k_apply_cells(MeshDesc m, const S *ub, const float *ublo, S *u0, float *u0lo,
                              S *u1, float *u1lo, const S *du, int ncc, double beta, double dt,
                              const double *dt_dev, const DevClock *clock) {
  if (clock && clock->done) return;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NP = (long long)m.nb * m.P;
  const long long n = (long long)b * m.P + cidx(m, k, j, i);
  const double h = dt_dev ? *dt_dev : dt;
  for (int v = 0; v < ncc; v++) {
    if (sizeof(S) == 4 && v == CENER) {
      const double eb = load_ener(ub, ublo, NP, n), e0 = load_ener(u0, u0lo, NP, n);
      const double e0n = beta * eb + (1.0 - beta) * e0;
      store_ener(u0, u0lo, NP, n, e0n);
      store_ener(u1, u1lo, NP, n, e0n + beta * h * double(du[v * NP + n]));
      continue;
    }
    const S bt = S(beta);
    const S x0 = bt * ub[v * NP + n] + (S(1.0) - bt) * u0[v * NP + n];
    u0[v * NP + n] = x0;
    u1[v * NP + n] = x0 + bt * S(h) * du[v * NP + n];
  }
}

// FluxDivergence then ApplyDuDt of the cell variables in one pass, for
// adaptive hydro meshes (which have no fused stage): the expressions and
// their order are those of k_flux_divergence and k_apply_cells, with dU/dt
// held in a register instead of the dUdt container.  One thread per (cell,
// variable): an adaptive mesh can hold fewer cells than the GPU has thread
// slots, and independent variables keep more loads in flight.
template <typename S>
__global__ void k_div_apply(MeshDesc m, const S *flux, const S *ub, const float *ublo, S *u0, float *u0lo, S *u1,
                            float *u1lo, int ncc, double beta, double dt, const double *dt_dev,
                            const DevClock *clock) {
  if (clock && clock->done) return;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf, NP = (long long)m.nb * m.P;
  const long long bo = (long long)b * m.Pf;
  const long long n = (long long)b * m.P + cidx(m, k, j, i);
  const double h = dt_dev ? *dt_dev : dt;
  const int v = blockIdx.y;
  S d = S(0);
  for (int dir = 0; dir < m.ndim; dir++) {
    const int kp = k + (dir == 2), jp = j + (dir == 1), ip = i + (dir == 0);
    const S A = S(blk_area(m, b, dir));
    const S *F = flux + ((long long)dir * ncc + v) * NF + bo;
    d -= (A * F[fidx(m, kp, jp, ip)] - A * F[fidx(m, k, j, i)]);
  }
  const S du = d / S(blk_vol(m, b));
  if (sizeof(S) == 4 && v == CENER) {
    const double eb = load_ener(ub, ublo, NP, n), e0 = load_ener(u0, u0lo, NP, n);
    const double e0n = beta * eb + (1.0 - beta) * e0;
    store_ener(u0, u0lo, NP, n, e0n);
    store_ener(u1, u1lo, NP, n, e0n + beta * h * double(du));
    return;
  }
  const S bt = S(beta);
  const S x0 = bt * ub[v * NP + n] + (S(1.0) - bt) * u0[v * NP + n];
  u0[v * NP + n] = x0;
  u1[v * NP + n] = x0 + bt * S(h) * du;
}

int launch_div_apply(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta, double dt,
                     const double *dt_dev) {
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  const DevClock *clk = dt_dev ? c->clock : nullptr;
  const dim3 grid(nblk(n), unsigned(c->ncc));
  if (c->esz == 8)
    k_div_apply<double><<<grid, kThreads, 0, c->stream>>>(
        m, (const double *)c->flux, (const double *)base.cc, nullptr, (double *)md0.cc, nullptr,
        (double *)md1.cc, nullptr, c->ncc, beta, dt, dt_dev, clk);
  else
    k_div_apply<float><<<grid, kThreads, 0, c->stream>>>(
        m, (const float *)c->flux, (const float *)base.cc, (const float *)base.ener_lo, (float *)md0.cc,
        (float *)md0.ener_lo, (float *)md1.cc, (float *)md1.ener_lo, c->ncc, beta, dt, dt_dev, clk);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "div_apply");
}

template <typename S>
__global__ void k_apply_faces(MeshDesc m, const S *fb, S *f0, S *f1, const S *df, int face,
                              double beta, double dt, const double *dt_dev, const DevClock *clock) {
  if (clock && clock->done) return;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int n0 = m.nx[0] + (face == 0), n1 = m.nx[1] + (face == 1), n2 = m.nx[2] + (face == 2);
  const long long per = (long long)n0 * n1 * n2;
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, n0, n1, b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf;
  const long long n = face * NF + (long long)b * m.Pf + fidx(m, k, j, i);
  const double h = dt_dev ? *dt_dev : dt;
  const S bt = S(beta);
  const S x0 = bt * fb[n] + (S(1.0) - bt) * f0[n];
  f0[n] = x0;
  f1[n] = x0 + bt * S(h) * df[n];
}

int launch_apply_dudt(kmy_ctx *c, Container &base, Container &md0, Container &md1,
                      Container &dudt, double beta, double dt, const double *dt_dev) {
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  const DevClock *clk = dt_dev ? c->clock : nullptr;
  if (c->esz == 8)
    k_apply_cells<double><<<nblk(n), kThreads, 0, c->stream>>>(
        m, (const double *)base.cc, nullptr, (double *)md0.cc, nullptr, (double *)md1.cc, nullptr,
        (const double *)dudt.cc, c->ncc, beta, dt, dt_dev, clk);
  else
    k_apply_cells<float><<<nblk(n), kThreads, 0, c->stream>>>(
        m, (const float *)base.cc, (const float *)base.ener_lo, (float *)md0.cc,
        (float *)md0.ener_lo, (float *)md1.cc, (float *)md1.ener_lo, (const float *)dudt.cc,
        c->ncc, beta, dt, dt_dev, clk);
  c->launches++;
  if (c->prm.mhd && m.ndim > 1) return launch_apply_faces(c, base, md0, md1, dudt, beta, dt, dt_dev);
  return cuda_check(c, cudaGetLastError(), "apply_dudt");
}

// The face-field half of ApplyDuDt for every active face direction.
int launch_apply_faces(kmy_ctx *c, Container &base, Container &md0, Container &md1, Container &dudt,
                       double beta, double dt, const double *dt_dev) {
  const MeshDesc &m = c->m;
  const DevClock *clk = dt_dev ? c->clock : nullptr;
  for (int face = 0; face < m.ndim; face++) {
    const long long nfc =
        (long long)(m.nx[0] + (face == 0)) * (m.nx[1] + (face == 1)) * (m.nx[2] + (face == 2)) * m.nb;
    if (c->esz == 8)
      k_apply_faces<double><<<nblk(nfc), kThreads, 0, c->stream>>>(
          m, (const double *)base.fc, (double *)md0.fc, (double *)md1.fc, (const double *)dudt.fc,
          face, beta, dt, dt_dev, clk);
    else
      k_apply_faces<float><<<nblk(nfc), kThreads, 0, c->stream>>>(
          m, (const float *)base.fc, (float *)md0.fc, (float *)md1.fc, (const float *)dudt.fc,
          face, beta, dt, dt_dev, clk);
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "apply_dudt");
}

// ---------------------------------------------------------------------------
// The face update of a constrained-transport stage in one kernel per face
// direction: each face's edge EMFs from the face fluxes (CalculateEMF's
// arithmetic average, as k_edge_emf), their Stokes sum (FluxStokes, as
// k_flux_stokes) and the low-storage update (ApplyDuDt, as k_apply_faces),
// with the same expressions in the same order, so EMFs and face values agree
// bit for bit with those three kernels.  The EMF and dU/dt arrays are not
// written.  Edges on block faces read the ghost-layer fluxes of k_flux_halo.

// Edge EMF of edge direction E at in-block face-array offset p: the
// arithmetic average of CalculateEMF, with k_edge_emf's expression.  Fa / Fb
// are the block's flux arrays of the two terms: E = 2 reads F_y[B_x] and
// F_x[B_y], E = 0 F_z[B_y] and F_y[B_z], E = 1 F_x[B_z] and F_z[B_x]; sa / sb
// are the face-array strides the terms shift along (i, j or k).
template <typename S>
__device__ __forceinline__ S edge_emf_at(const S *Fa, const S *Fb, unsigned p, unsigned sa, unsigned sb) {
  return S(1.0) * S(0.25) * (Fa[p - sa] + Fa[p] - Fb[p - sb] - Fb[p]);
}

template <typename S, int FACE>
__global__ void k_ct_faces(MeshDesc m, const S *flux, const S *fb, S *f0, S *f1, double beta,
                           const double *dt_dev, const DevClock *clock) {
  if (clock->done) return;
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int n0 = m.nx[0] + (FACE == 0), n1 = m.nx[1] + (FACE == 1), n2 = m.nx[2] + (FACE == 2);
  const long long per = (long long)n0 * n1 * n2;
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, n0, n1, b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf, bo = (long long)b * m.Pf;
  // in-block face-array offsets (a block's face arrays hold fewer than 2^32)
  const unsigned si = 1, sj = unsigned(m.nf[0]), sk = unsigned(m.nf[0]) * unsigned(m.nf[1]);
  const unsigned p = (unsigned(k) * unsigned(m.nf[1]) + unsigned(j)) * unsigned(m.nf[0]) + unsigned(i);
  auto Fp = [&](int dir, int bcomp) { return flux + ((long long)dir * 8 + CMAGC0 + bcomp) * NF + bo; };
  // The face's edges in FluxStokes order (grid_update.hpp:80-137): edge
  // direction, the axis its second EMF sits one node further along, and the
  // sign; in 2D only the z edges.
  auto stokes = [&](int edge, int axis) -> S {
    const unsigned sax = axis == 0 ? si : axis == 1 ? sj : sk;
    const S sign = ((axis + 1) % 3 == edge) ? S(1.0) : S(-1.0);
    const S L = S(blk_dx(m, b, edge));
    S Ea, Eb;
    if (edge == 2) {
      Ea = edge_emf_at(Fp(1, 0), Fp(0, 1), p, si, sj);
      Eb = edge_emf_at(Fp(1, 0), Fp(0, 1), p + sax, si, sj);
    } else if (edge == 0) {
      Ea = edge_emf_at(Fp(2, 1), Fp(1, 2), p, sj, sk);
      Eb = edge_emf_at(Fp(2, 1), Fp(1, 2), p + sax, sj, sk);
    } else {
      Ea = edge_emf_at(Fp(0, 2), Fp(2, 0), p, sk, si);
      Eb = edge_emf_at(Fp(0, 2), Fp(2, 0), p + sax, sk, si);
    }
    return sign * (L * Ea - L * Eb);
  };
  S out = S(0);
  if (FACE == 0) {
    out += stokes(2, 1);
    if (m.ndim > 2) out += stokes(1, 2);
  } else if (FACE == 1) {
    out += stokes(2, 0);
    if (m.ndim > 2) out += stokes(0, 2);
  } else {
    out += stokes(0, 1);
    out += stokes(1, 0);
  }
  out *= S(1.) / (S(blk_area(m, b, FACE)) + S(1.e-36));
  const long long n = FACE * NF + bo + p;
  const double h = *dt_dev;
  const S bt = S(beta);
  const S x0 = bt * fb[n] + (S(1.0) - bt) * f0[n];
  f0[n] = x0;
  f1[n] = x0 + bt * S(h) * out;
}

int launch_ct_faces(kmy_ctx *c, Container &base, Container &md0, Container &md1, double beta) {
  const MeshDesc &m = c->m;
  for (int f = 0; f < m.ndim; f++) {
    const long long nfc =
        (long long)(m.nx[0] + (f == 0)) * (m.nx[1] + (f == 1)) * (m.nx[2] + (f == 2)) * m.nb;
#define KMY_CTF(S_, F_)                                                                                    \
  k_ct_faces<S_, F_><<<nblk(nfc), kThreads, 0, c->stream>>>(m, (const S_ *)c->flux, (const S_ *)base.fc, \
                                                            (S_ *)md0.fc, (S_ *)md1.fc, beta,            \
                                                            &c->clock->dt, c->clock)
    if (c->esz == 8) {
      if (f == 0) KMY_CTF(double, 0);
      else if (f == 1) KMY_CTF(double, 1);
      else KMY_CTF(double, 2);
    } else {
      if (f == 0) KMY_CTF(float, 0);
      else if (f == 1) KMY_CTF(float, 1);
      else KMY_CTF(float, 2);
    }
#undef KMY_CTF
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "ct_faces");
}

// ---------------------------------------------------------------------------
// CT face -> cell average (primconsflux.cpp:102-129)
template <typename S>
__device__ __forceinline__ void face_average(const MeshDesc &m, const S *fc, int b, int k, int j,
                                             int i, S *B) {
  const long long NF = (long long)m.nb * m.Pf, bo = (long long)b * m.Pf;
  const S vol = S(blk_vol(m, b));
  const S a0 = S(blk_area(m, b, 0)), a1 = S(blk_area(m, b, 1)), a2 = S(blk_area(m, b, 2));
  if (m.ndim > 1) {
    B[0] = S(0.5) * S(blk_dx(m, b, 0)) *
           (a0 * fc[bo + fidx(m, k, j, i + 1)] + a0 * fc[bo + fidx(m, k, j, i)]) / vol;
    B[1] = S(0.5) * S(blk_dx(m, b, 1)) *
           (a1 * fc[NF + bo + fidx(m, k, j + 1, i)] + a1 * fc[NF + bo + fidx(m, k, j, i)]) / vol;
  }
  if (m.ndim > 2) {
    B[2] = S(0.5) * S(blk_dx(m, b, 2)) *
           (a2 * fc[2 * NF + bo + fidx(m, k + 1, j, i)] + a2 * fc[2 * NF + bo + fidx(m, k, j, i)]) / vol;
  }
}

// PreparePrimitive_impl (primconsflux.cpp:82-142) + EosWrapped(ener) (eos.cpp:71-103)
template <typename S, bool MHD>
__global__ void k_prepare_primitive(MeshDesc m, EosParams eos, S *cc, const float *lo, const S *fc,
                                    S *prim) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NP = (long long)m.nb * m.P;
  const long long n = (long long)b * m.P + cidx(m, k, j, i);
  S B[3] = {S(0), S(0), S(0)};
  if constexpr (MHD) {
    for (int d = 0; d < 3; d++) B[d] = cc[(CMAGC0 + d) * NP + n];
    face_average(m, fc, b, k, j, i, B);
    for (int d = 0; d < 3; d++) cc[(CMAGC0 + d) * NP + n] = B[d];
  }
  S V[MHD ? 10 : 7];
  Cons2PrimEos<MHD, S>(eos, cc[n], cc[CMOM0 * NP + n], cc[CMOM1 * NP + n], cc[CMOM2 * NP + n],
                       load_ener(cc, lo, NP, n), B, V);
  prim[PVEL0 * NP + n] = V[RVEL0];
  prim[PVEL1 * NP + n] = V[RVEL1];
  prim[PVEL2 * NP + n] = V[RVEL2];
  prim[PPRES * NP + n] = V[RPRES];
  prim[PBMOD * NP + n] = V[RBMOD];
  prim[PEINT * NP + n] = V[REINT];
  prim[PTEMP * NP + n] = kmax(S(0), V[REINT] / S(eos.cv));
}

int launch_prepare_primitive(kmy_ctx *c, Container &md1) {
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  if (c->esz == 8) {
    if (c->prm.mhd)
      k_prepare_primitive<double, true><<<nblk(n), kThreads, 0, c->stream>>>(
          m, c->eos, (double *)md1.cc, nullptr, (const double *)md1.fc, (double *)c->prim);
    else
      k_prepare_primitive<double, false><<<nblk(n), kThreads, 0, c->stream>>>(
          m, c->eos, (double *)md1.cc, nullptr, nullptr, (double *)c->prim);
  } else {
    if (c->prm.mhd)
      k_prepare_primitive<float, true><<<nblk(n), kThreads, 0, c->stream>>>(
          m, c->eos, (float *)md1.cc, (const float *)md1.ener_lo, (const float *)md1.fc, (float *)c->prim);
    else
      k_prepare_primitive<float, false><<<nblk(n), kThreads, 0, c->stream>>>(
          m, c->eos, (float *)md1.cc, (const float *)md1.ener_lo, nullptr, (float *)c->prim);
  }
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "prepare_primitive");
}

// ---------------------------------------------------------------------------
// EstimateTimeStep (hydro_time_step.cpp:19-64): min over interior cells and
// active directions of dx/(|v|+c_f); warp-shuffle min, one atomic per CTA on
// the bit pattern of a positive double (monotone as an unsigned integer).
__device__ __forceinline__ void atomic_min_pos_double(unsigned long long *addr, double v) {
  if (!(v >= 0.0)) v = 0.0;  // NaN/negative collapse to 0 -> flagged by the controller
  atomicMin(addr, (unsigned long long)__double_as_longlong(v));
}

__device__ __forceinline__ double block_min(double v) {
  __shared__ double wmin[32];
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wmin[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? wmin[lane] : INFINITY;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  }
  return v;
}

template <typename S, bool MHD>
__global__ void k_estimate_dt(MeshDesc m, const S *cc, const S *prim, DevClock *clock) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  double dtl = INFINITY;
  if (t < per * m.nb) {
    int b, i, j, k;
    unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
    i += m.g[0];
    j += m.g[1];
    k += m.g[2];
    const long long NP = (long long)m.nb * m.P;
    const long long n = (long long)b * m.P + cidx(m, k, j, i);
    S V[MHD ? 10 : 7];
    V[RDENS] = cc[n];
    V[RVEL0] = prim[PVEL0 * NP + n];
    V[RVEL1] = prim[PVEL1 * NP + n];
    V[RVEL2] = prim[PVEL2 * NP + n];
    V[RPRES] = prim[PPRES * NP + n];
    V[RBMOD] = prim[PBMOD * NP + n];
    V[REINT] = prim[PEINT * NP + n];
    if constexpr (MHD)
      for (int d = 0; d < 3; d++) V[RMAGC0 + d] = cc[(CMAGC0 + d) * NP + n];
    for (int dir = 0; dir < m.ndim; dir++) {
      const S cf = FastSpeed<MHD>(dir, V);
      const double x = double(S(blk_dx(m, b, dir)) / (fabs(V[RVEL0 + dir]) + cf));
      dtl = (x < dtl || x != x) ? x : dtl;
    }
  }
  dtl = block_min(dtl);
  if (threadIdx.x == 0) atomic_min_pos_double(&clock->dtmin_bits, dtl);
}

__global__ void k_reset_dtmin(DevClock *clock) { clock->dtmin_bits = 0x7FF0000000000000ull; }

int launch_estimate_dt(kmy_ctx *c, Container &md, bool reset) {
  const MeshDesc &m = c->m;
  if (reset) {
    k_reset_dtmin<<<1, 1, 0, c->stream>>>(c->clock);
    c->launches++;
  }
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  if (c->esz == 8) {
    if (c->prm.mhd)
      k_estimate_dt<double, true><<<nblk(n), kThreads, 0, c->stream>>>(m, (const double *)md.cc,
                                                                        (const double *)c->prim, c->clock);
    else
      k_estimate_dt<double, false><<<nblk(n), kThreads, 0, c->stream>>>(m, (const double *)md.cc,
                                                                         (const double *)c->prim, c->clock);
  } else {
    if (c->prm.mhd)
      k_estimate_dt<float, true><<<nblk(n), kThreads, 0, c->stream>>>(m, (const float *)md.cc,
                                                                       (const float *)c->prim, c->clock);
    else
      k_estimate_dt<float, false><<<nblk(n), kThreads, 0, c->stream>>>(m, (const float *)md.cc,
                                                                        (const float *)c->prim, c->clock);
  }
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "estimate_dt");
}

// Parthenon EvolutionDriver::SetGlobalTimeStep, restated (single thread).
__global__ void k_dt_controller(DevClock *clk, TimeParams tp, int mode, long long cells) {
  double dtmin;
  const unsigned long long bits = clk->dtmin_bits;
  dtmin = __longlong_as_double((long long)bits);
  const double big = 1.7976931348623157e308;
  if (mode == 2) {  // clamp the pending dt to a new tlim
    clk->done = clk->time >= tp.tlim;
    if (clk->time < tp.tlim && (tp.tlim - clk->time) < clk->dt) clk->dt = tp.tlim - clk->time;
    return;
  }
  if (mode == 0) {
    if (clk->done) return;
    advance_clock(clk, tp);
    clk->zone_cycles += (unsigned long long)cells;
    return;
  }
  if (mode == 3) {
    // after a remesh that followed mode 0: the new blocks' estimate also
    // bounds the next dt.  min(dt, est) clamped to tlim equals the mode-0
    // result over the union of both estimates.
    const double est = dtmin * tp.cfl_over_ndim;
    if (clk->status == 0 && (!(est > 0.0) || !(est < big))) clk->status = KMY_ERR_NONFINITE;
    clk->dt_est = fmin(clk->dt_est, est);
    double nd = fmin(clk->dt, est);
    if (clk->time < tp.tlim && (tp.tlim - clk->time) < nd) nd = tp.tlim - clk->time;
    clk->dt = nd;
    return;
  } else {
    clk->time = 0.0;
    clk->ncycle = 0;
    clk->zone_cycles = 0;
    clk->dt = big;
    clk->dt_taken = 0.0;
    clk->status = 0;
    clk->below_min = 0;
    clk->above_max = 0;
  }
  const double est = dtmin * tp.cfl_over_ndim;
  clk->dt_est = est;
  if (!(est > 0.0) || !(est < big)) clk->status = KMY_ERR_NONFINITE;
  double nd = clk->dt;
  if (nd < 0.1 * big) nd *= tp.dt_factor;
  nd = fmin(nd, est);
  if (clk->ncycle == 0) nd = fmin(nd, tp.dt_init);
  nd = fmin(nd, tp.dt_ceil);
  nd = fmin(nd, tp.dt_user);
  if (clk->time < tp.tlim && (tp.tlim - clk->time) < nd) nd = tp.tlim - clk->time;
  clk->dt = nd;
  clk->done = clk->time >= tp.tlim;
  clk->dtmin_bits = 0x7FF0000000000000ull;  // the next step's CFL minimum starts at +inf
}

int launch_dt_controller(kmy_ctx *c, int mode, long long cells) {
  const MeshDesc &m = c->m;
  if (cells < 0) cells = (long long)m.nb * m.nx[0] * m.nx[1] * m.nx[2];
  k_dt_controller<<<1, 1, 0, c->stream>>>(c->clock, c->prm.tp, mode, cells);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "dt_controller");
}

// ---------------------------------------------------------------------------
// FillDerived_impl (hydro.cpp:150-190): div B in FP64.
template <typename S>
__global__ void k_divb(MeshDesc m, const S *fc, double *divb) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NF = (long long)m.nb * m.Pf, bo = (long long)b * m.Pf;
  double d = 0.;
  for (int dir = 0; dir < m.ndim; dir++) {
    const int kp = k + (dir == 2), jp = j + (dir == 1), ip = i + (dir == 0);
    d += blk_area(m, b, dir) * double(fc[dir * NF + bo + fidx(m, kp, jp, ip)]) -
         blk_area(m, b, dir) * double(fc[dir * NF + bo + fidx(m, k, j, i)]);
  }
  divb[(long long)b * m.P + cidx(m, k, j, i)] = d / blk_vol(m, b);
}

int launch_fill_derived(kmy_ctx *c, Container &md) {
  if (!c->prm.mhd) return KMY_OK;
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  if (c->esz == 8)
    k_divb<double><<<nblk(n), kThreads, 0, c->stream>>>(m, (const double *)md.fc, c->divb);
  else
    k_divb<float><<<nblk(n), kThreads, 0, c->stream>>>(m, (const float *)md.fc, c->divb);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "fill_derived");
}

// ---------------------------------------------------------------------------
// eos.cpp:165-168, mode_init = dens_pres: sie = P/(gm1 rho), T, bulk modulus
template <typename S>
__global__ void k_eos_init(MeshDesc m, EosParams eos, const S *cc, S *prim) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NP = (long long)m.nb * m.P;
  const long long n = (long long)b * m.P + cidx(m, k, j, i);
  const S rho = cc[n];
  const S P = prim[PPRES * NP + n];
  const S gm1 = S(eos.gm1);
  const S sie = P / (gm1 * rho);
  prim[PEINT * NP + n] = sie;
  prim[PTEMP * NP + n] = kmax(S(0), sie / S(eos.cv));
  prim[PBMOD * NP + n] = kmax(S(0), (gm1 + S(1)) * gm1 * rho * sie);
}

int launch_eos_init(kmy_ctx *c, Container &md) {
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  if (c->esz == 8)
    k_eos_init<double><<<nblk(n), kThreads, 0, c->stream>>>(m, c->eos, (const double *)md.cc, (double *)c->prim);
  else
    k_eos_init<float><<<nblk(n), kThreads, 0, c->stream>>>(m, c->eos, (const float *)md.cc, (float *)c->prim);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "eos_init");
}

// ConvertToConserved_impl (primconsflux.cpp:19-79)
template <typename S, bool MHD>
__global__ void k_prim2cons(MeshDesc m, S *cc, float *lo, const S *fc, const S *prim) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  int b, i, j, k;
  unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
  i += m.g[0];
  j += m.g[1];
  k += m.g[2];
  const long long NP = (long long)m.nb * m.P;
  const long long n = (long long)b * m.P + cidx(m, k, j, i);
  S V[MHD ? 10 : 7], U[MHD ? 8 : 5];
  V[RDENS] = cc[n];
  V[RVEL0] = prim[PVEL0 * NP + n];
  V[RVEL1] = prim[PVEL1 * NP + n];
  V[RVEL2] = prim[PVEL2 * NP + n];
  V[RPRES] = prim[PPRES * NP + n];
  V[RBMOD] = prim[PBMOD * NP + n];
  V[REINT] = prim[PEINT * NP + n];
  if constexpr (MHD) {
    S B[3];
    for (int d = 0; d < 3; d++) B[d] = cc[(CMAGC0 + d) * NP + n];
    face_average(m, fc, b, k, j, i, B);
    for (int d = 0; d < 3; d++) V[RMAGC0 + d] = B[d];
  }
  Prim2Cons<MHD, S>(V, U);
  for (int v = 0; v < (MHD ? 8 : 5); v++) cc[v * NP + n] = U[v];
  if constexpr (sizeof(S) == 4) {
    // energy low word from an FP64 evaluation of the same sum
    const double d = double(V[RDENS]);
    double ek = 0.0, em = 0.0;
    for (int q = 0; q < 3; q++) ek += double(V[RVEL0 + q]) * double(V[RVEL0 + q]);
    if constexpr (MHD)
      for (int q = 0; q < 3; q++) em += double(V[RMAGC0 + q]) * double(V[RMAGC0 + q]);
    const double E = double(V[REINT]) * d + ek * (0.5 * d) + 0.5 * em;
    store_ener(cc, lo, NP, n, E);
  }
}

int launch_convert_to_conserved(kmy_ctx *c, Container &md) {
  const MeshDesc &m = c->m;
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  if (c->esz == 8) {
    if (c->prm.mhd)
      k_prim2cons<double, true><<<nblk(n), kThreads, 0, c->stream>>>(m, (double *)md.cc, nullptr,
                                                                     (const double *)md.fc, (const double *)c->prim);
    else
      k_prim2cons<double, false><<<nblk(n), kThreads, 0, c->stream>>>(m, (double *)md.cc, nullptr, nullptr,
                                                                      (const double *)c->prim);
  } else {
    if (c->prm.mhd)
      k_prim2cons<float, true><<<nblk(n), kThreads, 0, c->stream>>>(
          m, (float *)md.cc, (float *)md.ener_lo, (const float *)md.fc, (const float *)c->prim);
    else
      k_prim2cons<float, false><<<nblk(n), kThreads, 0, c->stream>>>(
          m, (float *)md.cc, (float *)md.ener_lo, nullptr, (const float *)c->prim);
  }
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "convert_to_conserved");
}

// ---------------------------------------------------------------------------
// Compensated FP64 sums (Neumaier) of the conserved variables times the cell
// volume over the interior.  Each CTA writes (sum, compensation) pairs; the
// host finishes the sum with the same compensated scheme.
constexpr int kSumBlocks = 592;

__device__ __forceinline__ void two_sum(double &s, double &c, double x) {
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

template <typename S>
__global__ void k_cons_sums(MeshDesc m, const S *cc, const float *lo, int ncc, double *part) {
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  const long long tot = per * m.nb;
  const long long NP = (long long)m.nb * m.P;
  __shared__ double ss[kThreads], sc[kThreads];
  for (int v = 0; v < ncc; v++) {
    double s = 0.0, cm = 0.0;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
      int b, i, j, k;
      unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
      i += m.g[0];
      j += m.g[1];
      k += m.g[2];
      const long long n = (long long)b * m.P + cidx(m, k, j, i);
      const double x = (v == CENER ? load_ener(cc, lo, NP, n) : double(cc[v * NP + n])) * blk_vol(m, b);
      two_sum(s, cm, x);
    }
    ss[threadIdx.x] = s;
    sc[threadIdx.x] = cm;
    __syncthreads();
    if (threadIdx.x == 0) {
      double S0 = 0.0, C0 = 0.0;
      for (int q = 0; q < blockDim.x; q++) {
        two_sum(S0, C0, ss[q]);
        C0 += sc[q];
      }
      part[(v * gridDim.x + blockIdx.x) * 2] = S0;
      part[(v * gridDim.x + blockIdx.x) * 2 + 1] = C0;
    }
    __syncthreads();
  }
}

int launch_conserved_sums(kmy_ctx *c, Container &md, double *out) {
  const MeshDesc &m = c->m;
  double *part = nullptr;
  const size_t bytes = sizeof(double) * 2 * kSumBlocks * c->ncc;
  int rc = cuda_check(c, cudaMallocAsync((void **)&part, bytes, c->stream), "sums alloc");
  if (rc) return rc;
  if (c->esz == 8)
    k_cons_sums<double><<<kSumBlocks, kThreads, 0, c->stream>>>(m, (const double *)md.cc, nullptr, c->ncc, part);
  else
    k_cons_sums<float><<<kSumBlocks, kThreads, 0, c->stream>>>(m, (const float *)md.cc,
                                                              (const float *)md.ener_lo, c->ncc, part);
  c->launches++;
  std::vector<double> h(2 * kSumBlocks * c->ncc);
  rc = cuda_check(c, cudaGetLastError(), "sums");
  if (!rc) rc = cuda_check(c, cudaMemcpyAsync(h.data(), part, bytes, cudaMemcpyDeviceToHost, c->stream), "sums copy");
  cudaFreeAsync(part, c->stream);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "sums sync");
  if (rc) return rc;
  for (int v = 0; v < c->ncc; v++) {
    double s = 0.0, cm = 0.0;
    for (int q = 0; q < kSumBlocks; q++) {
      const double x = h[(v * kSumBlocks + q) * 2];
      const double t = s + x;
      if (std::fabs(s) >= std::fabs(x)) cm += (s - t) + x;
      else cm += (x - t) + s;
      s = t;
      cm += h[(v * kSumBlocks + q) * 2 + 1];
    }
    out[v] = s + cm;
  }
  return KMY_OK;
}

// ErrorHistory (isentropic_vortex.hpp:150-200) on "base": sum |exact - have| * V
// over the area of the x1-x2 domain.
template <typename S>
__global__ void k_vortex_err(MeshDesc m, const S *cc, const S *prim, int var, int comp, double gamma,
                             double density, double pressure, double velx, double vely,
                             double strength, double mhd_strength, double *part) {
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  const long long tot = per * m.nb;
  const long long NP = (long long)m.nb * m.P;
  __shared__ double ss[kThreads];
  double s = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
       t += (long long)gridDim.x * blockDim.x) {
    int b, i, j, k;
    unflatten(t, per, m.nx[0], m.nx[1], b, i, j, k);
    const long long n = (long long)b * m.P + cidx(m, k + m.g[2], j + m.g[1], i + m.g[0]);
    const double x = m.xmin[0] + (double(blk_loc(m, b, 0) * m.nx[0] + i) + 0.5) * blk_dx(m, b, 0);
    const double y = m.xmin[1] + (double(blk_loc(m, b, 1) * m.nx[1] + j) + 0.5) * blk_dx(m, b, 1);
    const double r2 = x * x + y * y;
    const double dv = strength * exp(0.5 * (1.0 - r2)) / (2.0 * M_PI);
    const double T = pressure / density -
                     (gamma - 1.0) * strength * strength * exp(1.0 - r2) / (8.0 * gamma * M_PI * M_PI);
    double dens = pow(T, 1.0 / (gamma - 1.0));
    double presx = T * dens, Bx = 0.0, By = 0.0;
    if (mhd_strength >= 0.0) {  // StateMHD (isentropic_vortex.hpp:75-100)
      const double dB = mhd_strength * exp(0.5 * (1.0 - r2)) / (2.0 * M_PI);
      const double ex = exp(1.0 - r2);
      dens = 1.0;
      presx = pressure + (mhd_strength * mhd_strength / (8.0 * M_PI * M_PI)) * (1.0 - r2) * ex -
              (strength * strength / (8.0 * M_PI * M_PI)) * ex;
      Bx = -y * dB;
      By = +x * dB;
    }
    double exact, have;
    if (var == 3) {
      exact = comp == 0 ? Bx : comp == 1 ? By : 0.0;
      have = double(cc[(CMAGC0 + comp) * NP + n]);
    } else if (var == 0) {
      exact = dens;
      have = double(cc[n]);
    } else if (var == 1) {
      exact = comp == 0 ? velx - y * dv : comp == 1 ? vely + x * dv : 0.0;
      have = double(prim[(PVEL0 + comp) * NP + n]);
    } else {
      exact = presx;
      have = double(prim[PPRES * NP + n]);
    }
    s += fabs(exact - have) * blk_vol(m, b);
  }
  ss[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S0 = 0.0;
    for (int q = 0; q < blockDim.x; q++) S0 += ss[q];
    part[blockIdx.x] = S0;
  }
}

int launch_vortex_error(kmy_ctx *c, int var, int comp, double *out) {
  const MeshDesc &m = c->m;
  const Params &p = c->prm;
  double *part = nullptr;
  int rc = cuda_check(c, cudaMallocAsync((void **)&part, sizeof(double) * kSumBlocks, c->stream), "err alloc");
  if (rc) return rc;
  const Container &b = c->md["base"];
  const double dn = p.real("isentropic_vortex/density", 1.0), pr = p.real("isentropic_vortex/pressure", 1.0);
  const double vx = p.real("isentropic_vortex/velx", 1.0), vy = p.real("isentropic_vortex/vely", 1.0);
  const double st = p.real("isentropic_vortex/strength", 5.0);
  const double ms = p.mhd ? p.real("isentropic_vortex/mhd_strength", 1.0) : -1.0;
  if (c->esz == 8)
    k_vortex_err<double><<<kSumBlocks, kThreads, 0, c->stream>>>(m, (const double *)b.cc, (const double *)c->prim,
                                                                 var, comp, p.gamma, dn, pr, vx, vy, st, ms, part);
  else
    k_vortex_err<float><<<kSumBlocks, kThreads, 0, c->stream>>>(m, (const float *)b.cc, (const float *)c->prim,
                                                                var, comp, p.gamma, dn, pr, vx, vy, st, ms, part);
  c->launches++;
  std::vector<double> h(kSumBlocks);
  rc = cuda_check(c, cudaGetLastError(), "vortex err");
  if (!rc) rc = cuda_check(c, cudaMemcpyAsync(h.data(), part, sizeof(double) * kSumBlocks,
                                              cudaMemcpyDeviceToHost, c->stream), "err copy");
  cudaFreeAsync(part, c->stream);
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "err sync");
  if (rc) return rc;
  double s = 0.0;
  for (double x : h) s += x;
  const double area = (m.dx[0] * m.mesh_nx[0]) * (m.dx[1] * m.mesh_nx[1]);
  *out = s / area;
  return KMY_OK;
}

}  // namespace kmy

// kmy_fused.cuh -- one RK stage of the hydro update in a single launch.
//
// Each CTA owns a brick of interior cells of one meshblock.  For every active
// direction it stages the brick, extended by H cells along that direction,
// into shared memory as primitives (cons->prim + EOS on the fly), evaluates
// the face fluxes of that direction (reconstruction of all seven primitives at
// both cells of the face + Riemann solver), and accumulates the flux
// divergence of its own cells in registers.  The epilogue applies the
// low-storage RK update and, on the last stage, reduces the CFL time step.
//
// Ghost zones are not read: a halo cell is fetched from the interior of the
// block that owns it on the uniform mesh (periodic wrap, outflow clamp,
// reflect mirror with a sign flip), which is what the boundary exchange would
// have copied into the ghost zone.  The stage therefore reads U_stage once
// from HBM (halo re-reads hit L2), reads U_base for stages >= 2 and writes
// U_new, with no separate primitive, flux, dU/dt or ghost-exchange passes.
//
// Arithmetic per cell/face is the same as the per-task kernels
// (kmy_tasks.cu), which follow hydro_add_flux_tasks.cpp:36-264,
// grid_update.hpp:15-57, grid.cpp:213-241, primconsflux.cpp:82-142 and
// hydro_time_step.cpp:19-64.
#pragma once

#include <atomic>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

namespace kmy {

template <int NDIM, int RECON, bool MHD = false>
struct FusedShape {
  static constexpr int W = ReconWidth<RECON>::value;
  static constexpr int H = W + 1;
  static constexpr int B[3] = {NDIM == 3 ? 8 : NDIM == 2 ? 16 : 128, NDIM == 3 ? 8 : NDIM == 2 ? 16 : 1,
                               NDIM == 3 ? 8 : 1};
  // 3D MHD: 288 threads, so the 288 faces of a chunk's Riemann phase take
  // one round (at 256 one warp ran a second round alone)
  static constexpr int NT = (MHD && NDIM == 3) ? 288 : 256;
  static constexpr int NCELL = B[0] * B[1] * B[2];
  static constexpr int CPT = (NCELL + NT - 1) / NT;
  static constexpr int region(int d) { return (B[d] + 2 * H) * (NCELL / B[d]); }
  static constexpr int faces(int d) { return (B[d] + 1) * (NCELL / B[d]); }
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  static constexpr int REG_MAX =
      cmax(region(0), cmax(NDIM > 1 ? region(1) : 0, NDIM > 2 ? region(2) : 0));
  static constexpr int FACE_MAX =
      cmax(faces(0), cmax(NDIM > 1 ? faces(1) : 0, NDIM > 2 ? faces(2) : 0));
  // reconstructed variables: the hydro seven, plus the cell-centred field
  // with MHD (hydro_types.hpp:61-77 order)
  static constexpr int NR = MHD ? 10 : 7;
  // conserved components the stage updates from its fluxes: the hydro five,
  // plus B_z in 2D MHD (B_x, B_y and in 3D all of B come from the faces)
  static constexpr int NC = (MHD && NDIM == 2) ? 6 : 5;
  // conserved index of update slot v
  static constexpr int cons(int v) { return v < 5 ? v : CMAGC0 + 2; }
  // local coordinates per axis the brick's stencils touch
  static constexpr int TAB = cmax(B[0], cmax(B[1], B[2])) + 2 * H;
  // cells reconstructed per direction in the two-sided sweep: -1 .. B along d
  static constexpr int rcells(int d) { return (B[d] + 2) * (NCELL / B[d]); }
  static constexpr int RC_MAX = cmax(rcells(0), cmax(NDIM > 1 ? rcells(1) : 0, NDIM > 2 ? rcells(2) : 0));
  // Each cell is reconstructed once (both faces, shared smoothness
  // indicators) into shared memory and the Riemann problems read from there.
  // In 3D FP64 the transverse plane goes through in two chunks, which keeps
  // the reconstruction buffers small enough for two CTAs per SM; 3D FP32 MHD
  // (ten reconstructed variables) does the same for three.
  template <typename S>
  static constexpr int nchunk() {
    return (NDIM == 3 && (sizeof(S) == 8 || MHD)) ? 2 : 1;
  }
  // Face fluxes reuse the primitive tile with one chunk; with several they
  // need their own buffer (the tile is still being read).
  template <typename S>
  static constexpr int face_stride() {
    return nchunk<S>() == 1 ? NR * REG_MAX / NC : FACE_MAX;
  }
  template <typename S>
  static constexpr size_t smem_bytes() {
    const size_t rec = size_t(2 * NR) * (RC_MAX / nchunk<S>());
    const size_t flux = nchunk<S>() == 1 ? 0 : size_t(NC) * FACE_MAX;
    return sizeof(S) * (size_t(NR) * REG_MAX + rec + flux);
  }
};

template <typename S>
struct FusedArgs {
  MeshDesc m;
  EosParams eos;
  int limiter;
  const S *u0;
  const float *u0lo;
  const S *ub;
  const float *ublo;
  S *u1;
  float *u1lo;
  const S *prim;
  S *prim_out;  // primitives of u1's interior cells for the next stage (null: not kept)
  int stored;
  int last;
  double beta;
  DevClock *clock;
  int nbr[3];
  const S *fc0;  // MHD: face field of the stage input (the Riemann problems' normal B)
  S *flux;       // MHD: face fluxes for the edge EMFs, layout [dir][8][nb * Pf]
  int b0;        // first block of the launch (per-block launches; 0 when one launch covers the mesh)
};

// Global index -> interior index under the physical boundary of that side.
// The final clamp only matters for partial bricks far outside a tiny mesh;
// it keeps every access inside the mesh.
__device__ __forceinline__ int fz_map(int G, int N, int bc, bool &flip) {
  if (G >= 0 && G < N) return G;
  int M;
  if (bc == BC_PERIODIC) {
    M = ((G % N) + N) % N;
  } else if (bc == BC_OUTFLOW) {
    M = G < 0 ? 0 : N - 1;
  } else {
    flip = !flip;
    M = G < 0 ? -G - 1 : 2 * N - G - 1;
  }
  return M < 0 ? 0 : (M >= N ? N - 1 : M);
}

// Per-brick address tables.  The element offset of a mesh cell separates by
// axis: n = sum_d (owner_block_d * blocks_below_d * P + local_d * stride_d).
// For each axis and each local coordinate the brick can touch (o - H ..
// o + B + H - 1) the table holds that axis's share of n and whether the
// boundary map mirrored it (reflect), so staging a cell costs three shared
// loads instead of a boundary map and an integer division per axis.
template <int NDIM, int RECON>
struct FzTables {
  static constexpr int TAB = FusedShape<NDIM, RECON>::TAB;
  long long off[3][TAB];
  unsigned char flip[3][TAB];
};

template <typename S, int NDIM, int RECON>
__device__ __forceinline__ void fz_fill_tables(const FusedArgs<S> &a, const int lx[3], const int o[3],
                                               FzTables<NDIM, RECON> &t) {
  using Sh = FusedShape<NDIM, RECON>;
  constexpr int H = Sh::H;
  const MeshDesc &m = a.m;
  const int n0 = Sh::B[0] + 2 * H, n1 = Sh::B[1] + 2 * H, n2 = Sh::B[2] + 2 * H;
  for (int q = threadIdx.x; q < n0 + n1 + n2; q += Sh::NT) {
    const int d = q < n0 ? 0 : (q < n0 + n1 ? 1 : 2);
    const int i = q - (d == 0 ? 0 : d == 1 ? n0 : n0 + n1);
    const int l = o[d] + i - H;
    bool f = false;
    const int G = lx[d] * m.nx[d] + l;
    const int M = fz_map(G, m.mesh_nx[d], m.bc[d][G < 0 ? 0 : 1], f);
    const int ob = M / m.nx[d];
    const long long below = d == 0 ? 1 : d == 1 ? m.nbx[0] : (long long)m.nbx[0] * m.nbx[1];
    const long long stride = d == 0 ? 1 : d == 1 ? m.np[0] : (long long)m.np[0] * m.np[1];
    t.off[d][i] = ob * below * m.P + (long long)(M - ob * m.nx[d] + m.g[d]) * stride;
    t.flip[d][i] = f;
  }
}

// Primitive state of the mesh cell at element offset n (flips: mirrored axes).
template <typename S, bool MHD = false>
__device__ __forceinline__ void fz_load_prim(const FusedArgs<S> &a, long long n, const bool flip[3], S *V) {
  const MeshDesc &m = a.m;
  const long long NP = (long long)m.nb * m.P;
  const S dens = a.u0[n];
  // MHD: the cell-centred field (the face averages the previous stage left in
  // the conserved container); reflecting boundaries are not run with MHD
  S B[3] = {S(0), S(0), S(0)};
  if constexpr (MHD) {
#pragma unroll
    for (int d = 0; d < 3; d++) B[d] = a.u0[(CMAGC0 + d) * NP + n];
  }
  if (a.stored) {
    V[RDENS] = dens;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const S v = a.prim[(PVEL0 + d) * NP + n];
      V[RVEL0 + d] = flip[d] ? -v : v;
    }
    V[RPRES] = a.prim[PPRES * NP + n];
    V[RBMOD] = a.prim[PBMOD * NP + n];
    V[REINT] = a.prim[PEINT * NP + n];
    if constexpr (MHD) {
#pragma unroll
      for (int d = 0; d < 3; d++) V[RMAGC0 + d] = B[d];
    }
  } else {
    S mo[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const S v = a.u0[(CMOM0 + d) * NP + n];
      mo[d] = flip[d] ? -v : v;
    }
    double e = double(a.u0[CENER * NP + n]);
    if constexpr (sizeof(S) == 4) e += double(a.u0lo[n]);
    Cons2PrimEos<MHD, S>(a.eos, dens, mo[0], mo[1], mo[2], e, B, V);
  }
}

// 1. Primitives of the brick extended by H cells along DIR, into sp.
template <typename S, int NDIM, int RECON, int DIR, bool OVERLAP, bool MHD>
__device__ __forceinline__ void fz_stage_prims(const FusedArgs<S> &a, const FzTables<NDIM, RECON> &t, S *sp) {
  using Sh = FusedShape<NDIM, RECON, MHD>;
  constexpr int H = Sh::H;
  constexpr int E0 = Sh::B[0] + (DIR == 0 ? 2 * H : 0);
  constexpr int E1 = Sh::B[1] + (DIR == 1 ? 2 * H : 0);
  constexpr int E2 = Sh::B[2] + (DIR == 2 ? 2 * H : 0);
  constexpr int NREG = E0 * E1 * E2;
  constexpr int RM = Sh::REG_MAX;
  // Stored primitives with OVERLAP: every load of the thread's cells first,
  // then the stores, so the loads of all its cells are in flight together.
  // Otherwise one cell at a time: the conversion path (several FP64
  // equation-of-state evaluations at once would cost more registers than the
  // overlap saves) and the batched kernel, whose per-solve arguments already
  // hold many registers.
  constexpr int NIT = (NREG + Sh::NT - 1) / Sh::NT;
  auto cell = [&](int q, bool flip[3]) -> long long {
    // table index: region coordinate along DIR, brick coordinate + H across
    const int t0 = q % E0 + (DIR == 0 ? 0 : H);
    const int t1 = (q / E0) % E1 + (DIR == 1 ? 0 : H);
    const int t2 = q / (E0 * E1) + (DIR == 2 ? 0 : H);
    flip[0] = t.flip[0][t0] != 0;
    flip[1] = t.flip[1][t1] != 0;
    flip[2] = t.flip[2][t2] != 0;
    return t.off[0][t0] + t.off[1][t1] + t.off[2][t2];
  };
  if (OVERLAP && !MHD && a.stored) {
    const long long NP = (long long)a.m.nb * a.m.P;
    S V[NIT][7];
#pragma unroll
    for (int k = 0; k < NIT; k++) {
      const int q = threadIdx.x + k * Sh::NT;
      if (q < NREG) {
        bool flip[3];
        const long long n = cell(q, flip);
        V[k][RDENS] = a.u0[n];
#pragma unroll
        for (int d = 0; d < 3; d++) {
          const S v = a.prim[(PVEL0 + d) * NP + n];
          V[k][RVEL0 + d] = flip[d] ? -v : v;
        }
        V[k][RPRES] = a.prim[PPRES * NP + n];
        V[k][RBMOD] = a.prim[PBMOD * NP + n];
        V[k][REINT] = a.prim[PEINT * NP + n];
      }
    }
#pragma unroll
    for (int k = 0; k < NIT; k++) {
      const int q = threadIdx.x + k * Sh::NT;
      if (q < NREG) {
#pragma unroll
        for (int r = 0; r < 7; r++) sp[r * RM + q] = V[k][r];
      }
    }
  } else {
    for (int q = threadIdx.x; q < NREG; q += Sh::NT) {
      bool flip[3];
      const long long n = cell(q, flip);
      S V[Sh::NR];
      fz_load_prim<S, MHD>(a, n, flip, V);
#pragma unroll
      for (int r = 0; r < Sh::NR; r++) sp[r * RM + q] = V[r];
    }
  }
}

// Element offset of the brick's owned cell c, or -1 past the block's edge
// (partial bricks).
template <typename S, int NDIM, int RECON>
__device__ __forceinline__ long long fz_owned(const FusedArgs<S> &a, int b, const int o[3], int c) {
  using Sh = FusedShape<NDIM, RECON>;
  const MeshDesc &m = a.m;
  if (c >= Sh::NCELL) return -1;
  const int l0 = o[0] + c % Sh::B[0], l1 = o[1] + (c / Sh::B[0]) % Sh::B[1], l2 = o[2] + c / (Sh::B[0] * Sh::B[1]);
  if (l0 >= m.nx[0] || l1 >= m.nx[1] || l2 >= m.nx[2]) return -1;
  return (long long)b * m.P + ((long long)(l2 + m.g[2]) * m.np[1] + (l1 + m.g[1])) * m.np[0] + (l0 + m.g[0]);
}

// Ask L2 for the epilogue's inputs (U_base, and U_stage's momentum and
// energy, which the stored-primitive staging does not read) at the start of
// the stage, so the epilogue's loads do not wait on HBM.  One bulk prefetch
// per array and brick plane covers the plane's owned rows (the span from its
// first owned cell to its last, rounded out to 16 bytes; the rounding stays
// inside the block's ghost-padded storage).
template <typename S, int NDIM, int RECON, bool MHD>
__device__ __forceinline__ void fz_prefetch_epilogue(const FusedArgs<S> &a, int b, const int o[3]) {
  using Sh = FusedShape<NDIM, RECON, MHD>;
  constexpr int NV = Sh::NC;
  constexpr int NARR = 2 * NV + (sizeof(S) == 4 ? 2 : 0);
  const MeshDesc &m = a.m;
  const long long NP = (long long)m.nb * m.P;
  constexpr int B0 = Sh::B[0], B1 = Sh::B[1], B2 = Sh::B[2];
  const int len0 = min(B0, m.nx[0] - o[0]), len1 = min(B1, m.nx[1] - o[1]);
  for (int q = threadIdx.x; q < NARR * B2; q += Sh::NT) {
    const int arr = q / B2, l2 = o[2] + q % B2;
    if (l2 >= m.nx[2] || len0 <= 0 || len1 <= 0) continue;
    const long long n0 =
        (long long)b * m.P + ((long long)(l2 + m.g[2]) * m.np[1] + (o[1] + m.g[1])) * m.np[0] + (o[0] + m.g[0]);
    const long long n1 = n0 + (long long)(len1 - 1) * m.np[0] + len0;  // one past the plane's last owned cell
    uintptr_t lo, hi;
    if (arr < 2 * NV) {
      const S *base = arr < NV ? a.ub + Sh::cons(arr) * NP : a.u0 + Sh::cons(arr - NV) * NP;
      lo = uintptr_t(base + n0);
      hi = uintptr_t(base + n1);
    } else {
      const float *base = arr == 2 * NV ? a.ublo : a.u0lo;
      lo = uintptr_t(base + n0);
      hi = uintptr_t(base + n1);
    }
    lo &= ~uintptr_t(15);
    hi = (hi + 15) & ~uintptr_t(15);
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"(unsigned(hi - lo)) : "memory");
  }
}

// Last step of a direction: the divergence contribution of the DIR faces in sf
// to the owned cells' accumulators.
template <typename S, int NDIM, int RECON, int DIR, bool MHD>
__device__ __forceinline__ void fz_accumulate(const FusedArgs<S> &a, const S *sf,
                                              S (&du)[FusedShape<NDIM, RECON, MHD>::CPT][FusedShape<NDIM, RECON, MHD>::NC]) {
  using Sh = FusedShape<NDIM, RECON, MHD>;
  constexpr int B0 = Sh::B[0], B1 = Sh::B[1];
  constexpr int FM = Sh::template face_stride<S>();
  const S A = S(a.m.area[DIR]);
#pragma unroll
  for (int s = 0; s < Sh::CPT; s++) {
    const int c = threadIdx.x + s * Sh::NT;
    if (c < Sh::NCELL) {
      const int x = c % B0, y = (c / B0) % B1, z = c / (B0 * B1);
      int lo, hi;
      if (DIR == 0) {
        lo = x + (B0 + 1) * (y + B1 * z);
        hi = lo + 1;
      } else if (DIR == 1) {
        lo = x + B0 * (y + (B1 + 1) * z);
        hi = lo + B0;
      } else {
        lo = x + B0 * (y + B1 * z);
        hi = lo + B0 * B1;
      }
#pragma unroll
      for (int v = 0; v < Sh::NC; v++) du[s][v] -= (A * sf[v * FM + hi] - A * sf[v * FM + lo]);
    }
  }
}

// One direction, two-sided reconstruction: every cell from -1 to B along DIR
// is reconstructed once per primitive (both face values share the smoothness
// indicators and weights), one (primitive, cell) pair per thread so the
// CTA's threads stay busy; the Riemann solver then reads the two states of
// each face from shared memory.  The FP64 stage works through the
// transverse plane in NCH chunks so its reconstruction buffers stay small
// enough for two CTAs per SM; in FP32 one chunk covers the plane and the
// face fluxes reuse the primitive tile's storage.
template <typename S, int NDIM, int RECON, int RIEMANN, int DIR, bool OVERLAP, bool MHD>
__device__ __forceinline__ void fz_direction2(const FusedArgs<S> &a, const FzTables<NDIM, RECON> &tb, int b,
                                              const int o[3], unsigned short *rofs, S *sp, S *rm, S *rp, S *sf,
                                              S (&du)[FusedShape<NDIM, RECON, MHD>::CPT][FusedShape<NDIM, RECON, MHD>::NC]) {
  using Sh = FusedShape<NDIM, RECON, MHD>;
  constexpr int H = Sh::H, W = Sh::W;
  constexpr int B0 = Sh::B[0], B1 = Sh::B[1], B2 = Sh::B[2];
  constexpr int E0 = B0 + (DIR == 0 ? 2 * H : 0);
  constexpr int E1 = B1 + (DIR == 1 ? 2 * H : 0);
  constexpr int RM = Sh::REG_MAX;
  constexpr int NCH = Sh::template nchunk<S>();
  constexpr int RC = Sh::RC_MAX / NCH;
  constexpr int FM = Sh::template face_stride<S>();
  constexpr int ST = DIR == 0 ? 1 : DIR == 1 ? E0 : E0 * E1;  // region stride along DIR
  // the transverse axis split into chunks
  constexpr int CA = DIR == 2 ? 1 : 2;
  // reconstruction grid of one chunk: B+2 cells along DIR (positions -1 .. B)
  constexpr int C0 = B0 + (DIR == 0 ? 2 : 0);
  constexpr int C1 = (B1 + (DIR == 1 ? 2 : 0)) / (CA == 1 ? NCH : 1);
  constexpr int C2 = (B2 + (DIR == 2 ? 2 : 0)) / (CA == 2 ? NCH : 1);
  constexpr int NRC = C0 * C1 * C2;
  static_assert(NRC <= RC, "chunk exceeds the reconstruction buffers");
  static_assert(NCH == 1 || ((CA == 1 ? B1 : B2) % NCH == 0 && DIR != CA), "chunks must split a transverse axis");
  constexpr int RST = DIR == 0 ? 1 : DIR == 1 ? C0 : C0 * C1;  // chunk-grid stride along DIR
  // faces: B+1 along DIR; of one chunk and of the whole brick
  constexpr int F0 = DIR == 0 ? B0 + 1 : B0, F1 = DIR == 1 ? B1 + 1 : B1;
  constexpr int G0 = F0, G1 = CA == 1 ? F1 / NCH : F1;
  constexpr int G2 = (DIR == 2 ? B2 + 1 : B2) / (CA == 2 ? NCH : 1);
  constexpr int NFC = G0 * G1 * G2;
  const int tid = threadIdx.x;

  // FP32 reconstructs two cells per thread in packed arithmetic, (r, q) and
  // (r, q + NRC/2).  The chunk's grid is halved along its slowest axis of
  // extent > 1, so the partner's region cell lies a constant PO further.
  // rofs holds the region offset of each cell q of the first half of chunk 0;
  // chunk ch adds its origin's offset.
  constexpr int PA = C2 > 1 ? 2 : (C1 > 1 ? 1 : 0);
  constexpr int HALF = NRC / 2;
  constexpr int PO = PA == 2 ? (C2 / 2) * E0 * E1 : PA == 1 ? (C1 / 2) * E0 : C0 / 2;
  if constexpr (sizeof(S) == 4) {
    static_assert((PA == 2 ? C2 : PA == 1 ? C1 : C0) % 2 == 0, "pairs split an even axis of the chunk");
    static_assert(Sh::REG_MAX < 65536, "region offsets are 16-bit");
    for (int q = tid; q < HALF; q += Sh::NT) {
      const int x = q % C0, y = (q / C0) % C1, z = q / (C0 * C1);
      // region coordinate: position p = x - 1 along DIR sits at p + H
      const int ex = x + (DIR == 0 ? H - 1 : 0), ey = y + (DIR == 1 ? H - 1 : 0), ez = z + (DIR == 2 ? H - 1 : 0);
      rofs[q] = (unsigned short)(ex + E0 * (ey + E1 * ez));
    }
  }
  fz_stage_prims<S, NDIM, RECON, DIR, OVERLAP, MHD>(a, tb, sp);
  __syncthreads();

#pragma unroll 1
  for (int ch = 0; ch < NCH; ch++) {
    const int c1 = CA == 1 ? ch * C1 : 0, c2 = CA == 2 ? ch * C2 : 0;
    // 2. both face values of every (primitive, cell) of the chunk
    if constexpr (sizeof(S) == 4) {
      // item it = r * HALF + q, stepping by NT without divisions
      const S *sc = sp + E0 * (c1 + E1 * c2);  // the chunk's origin in the region
      int r = tid / HALF, q = tid - (tid / HALF) * HALF;
#pragma unroll 2
      for (; r < Sh::NR;) {
        const S *c = sc + r * RM + rofs[q];
        float2 s[5];
#pragma unroll
        for (int k = 0; k < 5; k++)
          s[k] = (k - 2 >= -W && k - 2 <= W) ? make_float2(c[(k - 2) * ST], c[(k - 2) * ST + PO]) : p2(0.f);
        float2 vm, vp;
        ReconstructBoth2<RECON>(a.limiter, s, vm, vp);
        rm[r * RC + q] = vm.x;
        rm[r * RC + q + HALF] = vm.y;
        rp[r * RC + q] = vp.x;
        rp[r * RC + q + HALF] = vp.y;
        q += Sh::NT % HALF;
        r += Sh::NT / HALF;
        if (q >= HALF) {
          q -= HALF;
          r++;
        }
      }
    } else {
      for (int it = tid; it < Sh::NR * NRC; it += Sh::NT) {
        const int r = it / NRC, q = it - r * NRC;
        const int x = q % C0, y = (q / C0) % C1 + c1, z = q / (C0 * C1) + c2;
        // region coordinate: position p = x - 1 along DIR sits at p + H
        const int ex = x + (DIR == 0 ? H - 1 : 0), ey = y + (DIR == 1 ? H - 1 : 0), ez = z + (DIR == 2 ? H - 1 : 0);
        const S *c = sp + r * RM + ex + E0 * (ey + E1 * ez);
        S s[5];
#pragma unroll
        for (int k = 0; k < 5; k++) s[k] = (k - 2 >= -W && k - 2 <= W) ? c[(k - 2) * ST] : S(0);
        S vm, vp;
        if constexpr (RECON == WENOZ) {
          WenoZBothTwoDiv<S>(s, vm, vp);
        } else {
          Reconstruct<RECON, S>(a.limiter, s, vm, vp);
        }
        rm[r * RC + q] = vm;
        rp[r * RC + q] = vp;
      }
    }
    __syncthreads();

    // 3. Riemann flux at the chunk's DIR faces; the face at position f joins
    // reconstruction cells f (its low cell, position f-1) and f+1.
    // MHD: the face (x, y, z) of the chunk's face grid sits at block-local
    // cell coordinates L (the face between cells L-1 and L along DIR); its
    // offset in the face arrays, clamped into the block for faces of partial
    // bricks (which no owned cell uses), and whether this brick writes its
    // flux for the edge EMFs (each interior face once).
    auto face_at = [&](int x, int y, int z, long long &fo) -> bool {
      const MeshDesc &m = a.m;
      const int L[3] = {o[0] + x, o[1] + y + c1, o[2] + z + c2};
      constexpr int BD = DIR == 0 ? B0 : DIR == 1 ? B1 : B2;
      bool own = L[DIR] <= m.nx[DIR] && (L[DIR] - o[DIR] < BD || L[DIR] == m.nx[DIR]);
      int c[3];
#pragma unroll
      for (int t = 0; t < 3; t++) {
        const int hi = m.nx[t] - (t == DIR ? 0 : 1);
        if (t != DIR) own = own && L[t] <= hi;
        c[t] = min(L[t], hi);
      }
      fo = (long long)b * m.Pf + ((long long)(c[2] + m.g[2]) * m.nf[1] + (c[1] + m.g[1])) * m.nf[0] + (c[0] + m.g[0]);
      return own;
    };
    // FP32 hydro pairs faces across the slowest transverse axis of even
    // extent (none in 1D); the partner lies LQO further in the
    // reconstruction grid and GFO further in the face grid.  (A packed MHD
    // HLL solver measured slower than the scalar one: more registers, one
    // CTA per SM fewer.)
    constexpr int QA = (sizeof(S) != 4 || MHD) ? -1
                       : (G2 > 1 && G2 % 2 == 0) ? 2
                       : (G1 > 1 && G1 % 2 == 0) ? 1
                       : (G0 % 2 == 0 && DIR != 0) ? 0 : -1;
    if constexpr (QA >= 0) {
      static_assert(QA != DIR, "faces pair across a transverse axis");
      constexpr int H0 = QA == 0 ? G0 / 2 : G0, H1 = QA == 1 ? G1 / 2 : G1, H2 = QA == 2 ? G2 / 2 : G2;
      constexpr int LQO = QA == 0 ? G0 / 2 : QA == 1 ? (G1 / 2) * C0 : (G2 / 2) * C0 * C1;
      constexpr int GFO = QA == 0 ? G0 / 2 : QA == 1 ? (G1 / 2) * F0 : (G2 / 2) * F0 * F1;
      for (int it = tid; it < H0 * H1 * H2; it += Sh::NT) {
        const int x = it % H0, y = (it / H0) % H1, z = it / (H0 * H1);
        const int lq = x + C0 * (y + C1 * z);
        float2 vL[7], vR[7];
#pragma unroll
        for (int r = 0; r < 7; r++) {
          vL[r] = make_float2(rp[r * RC + lq], rp[r * RC + lq + LQO]);
          vR[r] = make_float2(rm[r * RC + lq + RST], rm[r * RC + lq + RST + LQO]);
        }
        float2 F[5];
        RiemannFlux2<RIEMANN, DIR>(vL, vR, F);
        const int gf = x + F0 * ((y + c1) + F1 * (z + c2));
#pragma unroll
        for (int v = 0; v < 5; v++) {
          sf[v * FM + gf] = F[v].x;
          sf[v * FM + gf + GFO] = F[v].y;
        }
      }
    } else {
      for (int it = tid; it < NFC; it += Sh::NT) {
        const int x = it % G0, y = (it / G0) % G1, z = it / (G0 * G1);
        const int lq = x + C0 * (y + C1 * z);
        S vL[Sh::NR], vR[Sh::NR];
#pragma unroll
        for (int r = 0; r < Sh::NR; r++) {
          vL[r] = rp[r * RC + lq];
          vR[r] = rm[r * RC + lq + RST];
        }
        long long fo = 0;
        bool own = false;
        if constexpr (MHD) {
          own = face_at(x, y, z, fo);
          // CT: the normal component is the face field (hydro_add_flux_tasks.cpp:343-346)
          const S bn = a.fc0[(long long)DIR * a.m.nb * a.m.Pf + fo];
          vL[RMAGC0 + DIR] = bn;
          vR[RMAGC0 + DIR] = bn;
        }
        S F[MHD ? 8 : 5];
        RiemannFlux<RIEMANN, MHD, DIR, S>(vL, vR, F);
        const int gf = x + F0 * ((y + c1) + F1 * (z + c2));
#pragma unroll
        for (int v = 0; v < Sh::NC; v++) sf[v * FM + gf] = F[Sh::cons(v)];
        if constexpr (MHD) {
          // the transverse field fluxes the edge EMFs read
          if (own) {
            const long long NF = (long long)a.m.nb * a.m.Pf;
#pragma unroll
            for (int t = 0; t < NDIM; t++)
              if (t != DIR) a.flux[((long long)DIR * 8 + CMAGC0 + t) * NF + fo] = F[CMAGC0 + t];
          }
        }
      }
    }
    __syncthreads();
  }

  fz_accumulate<S, NDIM, RECON, DIR, MHD>(a, sf, du);
  __syncthreads();
}

// Brick br of block b for one stage: the whole per-CTA body.  Every thread of
// the CTA calls it (it synchronises internally).
template <typename S, int NDIM, int RECON, int RIEMANN, bool OVERLAP, bool MHD = false>
__device__ __forceinline__ void fused_brick(const FusedArgs<S> &a, int b, int br, double dt) {
  using Sh = FusedShape<NDIM, RECON, MHD>;
  constexpr int NV = Sh::NC;
  extern __shared__ __align__(16) unsigned char kmy_smem[];
  S *sp = reinterpret_cast<S *>(kmy_smem);

  const MeshDesc &m = a.m;
  const int o[3] = {(br % a.nbr[0]) * Sh::B[0], ((br / a.nbr[0]) % a.nbr[1]) * Sh::B[1],
                    (br / (a.nbr[0] * a.nbr[1])) * Sh::B[2]};
  const int lx[3] = {b % m.nbx[0], (b / m.nbx[0]) % m.nbx[1], b / (m.nbx[0] * m.nbx[1])};

  S du[Sh::CPT][NV];
#pragma unroll
  for (int s = 0; s < Sh::CPT; s++)
#pragma unroll
    for (int v = 0; v < NV; v++) du[s][v] = S(0);

  fz_prefetch_epilogue<S, NDIM, RECON, MHD>(a, b, o);
  __shared__ FzTables<NDIM, RECON> tb;
  fz_fill_tables<S, NDIM, RECON>(a, lx, o, tb);
  __syncthreads();
  constexpr int NCH = Sh::template nchunk<S>();
  S *rm = sp + Sh::NR * Sh::REG_MAX;
  S *rp = rm + Sh::NR * (Sh::RC_MAX / NCH);
  S *sf = NCH == 1 ? sp : rp + Sh::NR * (Sh::RC_MAX / NCH);
  __shared__ unsigned short rofs[sizeof(S) == 4 ? Sh::RC_MAX / 2 : 1];
  fz_direction2<S, NDIM, RECON, RIEMANN, 0, OVERLAP, MHD>(a, tb, b, o, rofs, sp, rm, rp, sf, du);
  if constexpr (NDIM > 1) fz_direction2<S, NDIM, RECON, RIEMANN, 1, OVERLAP, MHD>(a, tb, b, o, rofs, sp, rm, rp, sf, du);
  if constexpr (NDIM > 2) fz_direction2<S, NDIM, RECON, RIEMANN, 2, OVERLAP, MHD>(a, tb, b, o, rofs, sp, rm, rp, sf, du);

  // epilogue: low-storage update of the owned interior cells.  With OVERLAP
  // the inputs of all the thread's cells are loaded first so their loads
  // overlap; the batched kernel loads cell by cell.
  const long long NP = (long long)m.nb * m.P;
  const S vol = S(m.vol);
  const S bt = S(a.beta);
  double dtl = INFINITY;
  struct In {
    long long n;
    S b[NV], z[NV];
    float blo, zlo;
  };
  auto load = [&](int s, In &in) {
    in.n = fz_owned<S, NDIM, RECON>(a, b, o, threadIdx.x + s * Sh::NT);
    if (in.n < 0) return;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      in.b[v] = a.ub[Sh::cons(v) * NP + in.n];
      in.z[v] = a.u0[Sh::cons(v) * NP + in.n];
    }
    if constexpr (sizeof(S) == 4) {
      in.blo = a.ublo[in.n];
      in.zlo = a.u0lo[in.n];
    }
  };
  In pre[OVERLAP ? Sh::CPT : 1];
  if constexpr (OVERLAP) {
#pragma unroll
    for (int s = 0; s < Sh::CPT; s++) load(s, pre[s]);
  }
#pragma unroll
  for (int s = 0; s < Sh::CPT; s++) {
    In cur;
    if constexpr (OVERLAP) {
      cur = pre[s];
    } else {
      load(s, cur);
    }
    const long long n = cur.n;
    if (n < 0) continue;
    S un[NV];
    float unlo = 0.f;
#pragma unroll
    for (int v = 0; v < NV; v++) {
      const S dudt = du[s][v] / vol;
      if (sizeof(S) == 4 && v == CENER) {
        double eb = double(cur.b[CENER]), e0 = double(cur.z[CENER]);
        if constexpr (sizeof(S) == 4) {
          eb += double(cur.blo);
          e0 += double(cur.zlo);
        }
        const double e1 = (a.beta * eb + (1.0 - a.beta) * e0) + a.beta * dt * double(dudt);
        const float hi = float(e1);
        unlo = float(e1 - double(hi));
        a.u1[CENER * NP + n] = S(hi);
        if constexpr (sizeof(S) == 4) a.u1lo[n] = unlo;
        un[v] = S(hi);
        continue;
      }
      const S y0 = bt * cur.b[v] + (S(1.0) - bt) * cur.z[v];
      un[v] = y0 + bt * S(dt) * dudt;
      a.u1[Sh::cons(v) * NP + n] = un[v];
    }
    // MHD: the primitives and the time step wait for the face update
    if (!MHD && (a.last || a.prim_out)) {
      double e = double(un[CENER]);
      if constexpr (sizeof(S) == 4) e += double(unlo);
      S V[7];
      Cons2PrimEos<false, S>(a.eos, un[CDENS], un[CMOM0], un[CMOM1], un[CMOM2], e, nullptr, V);
      if (a.prim_out) {
        // the next stage stages these instead of converting its input again
#pragma unroll
        for (int d = 0; d < 3; d++) a.prim_out[(PVEL0 + d) * NP + n] = V[RVEL0 + d];
        a.prim_out[PPRES * NP + n] = V[RPRES];
        a.prim_out[PBMOD * NP + n] = V[RBMOD];
        a.prim_out[PEINT * NP + n] = V[REINT];
      }
      if (a.last) {
#pragma unroll
        for (int dir = 0; dir < NDIM; dir++) {
          const S cf = FastSpeed<false>(dir, V);
          double xv = double(S(m.dx[dir]) / (fabs(V[RVEL0 + dir]) + cf));
          if (xv != xv) xv = 0.0;
          dtl = xv < dtl ? xv : dtl;
        }
      }
    }
  }
  if (a.last) {
    for (int q = 16; q > 0; q >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, q));
    __shared__ double wmin[Sh::NT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) wmin[warp] = dtl;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = wmin[0];
      for (int w = 1; w < Sh::NT / 32; w++) v = fmin(v, wmin[w]);
      if (!(v >= 0.0)) v = 0.0;
      atomicMin(&a.clock->dtmin_bits, (unsigned long long)__double_as_longlong(v));
    }
  }
}

// A stage after the run reached tlim (queued ahead of the host's check)
// leaves the state as it is: u1 and the output primitives become copies of
// the input, so the host's container and buffer swaps stay consistent.
template <typename S, int NDIM, int RECON, bool MHD>
__device__ __forceinline__ void fused_passthrough(const FusedArgs<S> &a, int b, int br) {
  using Sh = FusedShape<NDIM, RECON>;
  constexpr int NCC = MHD ? 8 : 5;
  const MeshDesc &m = a.m;
  const long long NP = (long long)m.nb * m.P;
  const int o[3] = {(br % a.nbr[0]) * Sh::B[0], ((br / a.nbr[0]) % a.nbr[1]) * Sh::B[1],
                    (br / (a.nbr[0] * a.nbr[1])) * Sh::B[2]};
  for (int c = threadIdx.x; c < Sh::NCELL; c += Sh::NT) {
    const int l0 = o[0] + c % Sh::B[0], l1 = o[1] + (c / Sh::B[0]) % Sh::B[1], l2 = o[2] + c / (Sh::B[0] * Sh::B[1]);
    if (l0 >= m.nx[0] || l1 >= m.nx[1] || l2 >= m.nx[2]) continue;
    const long long n = (long long)b * m.P +
                        ((long long)(l2 + m.g[2]) * m.np[1] + (l1 + m.g[1])) * m.np[0] + (l0 + m.g[0]);
    if (a.u1 != a.u0) {
#pragma unroll
      for (int v = 0; v < NCC; v++) a.u1[v * NP + n] = a.u0[v * NP + n];
      if constexpr (sizeof(S) == 4) a.u1lo[n] = a.u0lo[n];
    }
    if (a.prim_out) {
      const bool keep[3] = {false, false, false};
      S V[7];
      fz_load_prim<S>(a, n, keep, V);
#pragma unroll
      for (int d = 0; d < 3; d++) a.prim_out[(PVEL0 + d) * NP + n] = V[RVEL0 + d];
      a.prim_out[PPRES * NP + n] = V[RPRES];
      a.prim_out[PBMOD * NP + n] = V[RBMOD];
      a.prim_out[PEINT * NP + n] = V[REINT];
    }
  }
}

// One stage of one mesh: one CTA per brick.
template <typename S, int NDIM, int RECON, int RIEMANN, bool MHD>
__global__ void __launch_bounds__(FusedShape<NDIM, RECON, MHD>::NT) k_fused_stage(FusedArgs<S> a) {
  const int nbrick = a.nbr[0] * a.nbr[1] * a.nbr[2];
  const int bl = blockIdx.x / nbrick, b = a.b0 + bl;
  if (a.clock->done) {
    fused_passthrough<S, NDIM, RECON, MHD>(a, b, blockIdx.x - bl * nbrick);
    return;
  }
  fused_brick<S, NDIM, RECON, RIEMANN, true, MHD>(a, b, blockIdx.x - bl * nbrick, a.clock->dt);
}

// ---------------------------------------------------------------------------
// Batched stage over many independent solves of one kernel class (precision,
// dimensionality, reconstruction, Riemann solver).  The work list is
// (solve, block, brick) with per-solve offsets prefix[]; a persistent grid
// strides over it.  The list, its length and every solve's clock live in
// device memory, so the same launch (and a CUDA graph of it) serves any mix.
template <typename S>
struct SolveDesc {
  MeshDesc m;
  EosParams eos;
  TimeParams tp;
  int limiter;
  int nstages;
  int nlim;       // steps after which the solve is done (< 0: none)
  int stored;     // stage 1 of the next step reads stored primitives (cleared by the controller)
  S *cont[3];     // containers "base", "1", "2"
  float *lo[3];   // their FP32 energy low words (FP32 only)
  const S *prim;
  double beta[3];
  DevClock *clock;
  int nbr[3];
};

template <typename S>
__device__ __forceinline__ void batch_args(const SolveDesc<S> &q, int stage, FusedArgs<S> &a) {
  // stage names base, 1, ..., nstages-1, base (Parthenon low-storage integrators)
  const int i0 = stage - 1, i1 = stage == q.nstages ? 0 : stage;
  a.m = q.m;
  a.eos = q.eos;
  a.limiter = q.limiter;
  a.u0 = q.cont[i0];
  a.u0lo = q.lo[i0];
  a.ub = q.cont[0];
  a.ublo = q.lo[0];
  a.u1 = q.cont[i1];
  a.u1lo = q.lo[i1];
  a.prim = q.prim;
  a.prim_out = nullptr;
  a.stored = stage == 1 ? q.stored : 0;
  a.last = stage == q.nstages;
  a.beta = q.beta[stage - 1];
  a.clock = q.clock;
  a.nbr[0] = q.nbr[0];
  a.nbr[1] = q.nbr[1];
  a.nbr[2] = q.nbr[2];
  a.fc0 = nullptr;
  a.flux = nullptr;
}

template <typename S, int NDIM, int RECON, int RIEMANN>
__global__ void __launch_bounds__(FusedShape<NDIM, RECON>::NT, sizeof(S) == 4 ? 3 : 2) k_fused_batch(const SolveDesc<S> *__restrict__ d,
                                                     const long long *__restrict__ prefix,
                                                     const int *nsolves_dev, int stage) {
  __shared__ FusedArgs<S> sa;
  __shared__ long long s_base;
  __shared__ int s_skip;
  __shared__ double s_dt;
  const int ns = *nsolves_dev;
  if (ns <= 0) return;
  const long long total = prefix[ns];
  for (long long w = blockIdx.x; w < total; w += gridDim.x) {
    if (threadIdx.x == 0) {
      int lo = 0, hi = ns - 1;  // last solve whose offset is <= w
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= w) lo = mid;
        else hi = mid - 1;
      }
      const SolveDesc<S> &q = d[lo];
      s_base = prefix[lo];
      s_skip = q.clock->done || stage > q.nstages;
      s_dt = q.clock->dt;
      batch_args(q, stage, sa);
    }
    __syncthreads();
    if (!s_skip) {
      const long long wl = w - s_base;
      const int nbrick = sa.nbr[0] * sa.nbr[1] * sa.nbr[2];
      const int b = int(wl / nbrick);
      fused_brick<S, NDIM, RECON, RIEMANN, false>(sa, b, int(wl - (long long)b * nbrick), s_dt);
    }
    __syncthreads();
  }
}

template <typename S, int NDIM, int RECON, int RIEMANN, bool MHD>
int fused_launch(kmy_ctx *c, FusedArgs<S> a) {
  using Sh = FusedShape<NDIM, RECON, MHD>;
  const MeshDesc &m = c->m;
  for (int d = 0; d < 3; d++) a.nbr[d] = (m.nx[d] + Sh::B[d] - 1) / Sh::B[d];
  const long long grid = (long long)a.nbr[0] * a.nbr[1] * a.nbr[2] * m.nb;
  const size_t smem = Sh::template smem_bytes<S>();
  auto kern = k_fused_stage<S, NDIM, RECON, RIEMANN, MHD>;
  // the shared-memory opt-in once per device and kernel, so a stream capture
  // (kmy_evolve's graphs) sees launches only
  static std::atomic<unsigned> opted{0};
  const unsigned bit = c->device < 32 ? 1u << c->device : 0u;
  if (!bit || !(opted.load() & bit)) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return cuda_check(c, e, "fused smem attribute");
    opted.fetch_or(bit);
  }
  if (c->prm.per_block && !MHD) {
    // one launch per meshblock, as a caller that steps blocks one at a time would
    const int per = a.nbr[0] * a.nbr[1] * a.nbr[2];
    for (int b = 0; b < m.nb; b++) {
      a.b0 = b;
      kern<<<unsigned(per), Sh::NT, smem, c->stream>>>(a);
      c->launches++;
    }
    return cuda_check(c, cudaGetLastError(), "fused stage");
  }
  a.b0 = 0;
  kern<<<unsigned(grid), Sh::NT, smem, c->stream>>>(a);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "fused stage");
}

// Hydro in 1D-3D; MHD (constrained transport) in 2D and 3D.
template <typename S>
int fused_dispatch(kmy_ctx *c, FusedArgs<S> a) {
  const int nd = c->m.ndim, rec = c->prm.recon, rie = c->prm.riemann;
  const bool mhd = c->prm.mhd;
#define KMY_FZ(ND, RC, M)                                            \
  if (nd == ND && rec == RC && mhd == M) {                           \
    return rie == HLL ? fused_launch<S, ND, RC, HLL, M>(c, a)        \
                      : fused_launch<S, ND, RC, HLLC, M>(c, a);      \
  }
#define KMY_FZ_ND(ND, M) KMY_FZ(ND, FOG, M) KMY_FZ(ND, PLM, M) KMY_FZ(ND, PPM, M) KMY_FZ(ND, WENOZ, M)
  KMY_FZ_ND(1, false)
  KMY_FZ_ND(2, false)
  KMY_FZ_ND(3, false)
  KMY_FZ_ND(2, true)
  KMY_FZ_ND(3, true)
#undef KMY_FZ_ND
#undef KMY_FZ
  c->err = "no fused kernel for this configuration";
  return KMY_ERR_BAD_PARAM;
}

}  // namespace kmy

// kmy_slab.cuh -- one RK stage of 3D hydro in FP32, streamed through each
// meshblock along z with TMA-staged plane pairs.
//
// Work item: one meshblock b and one tile of TY = 16 rows (y) by the block's
// full 32-cell width (x).  A persistent grid (one CTA of 512 threads per SM)
// strides over the (block, tile) work list.  Thread t owns the column
// (x = t % 32, y = oy + t / 32) and walks it along z two planes at a time, so
// every FP32 operation of the z sweep works on a float2 of planes (k, k+1)
// (sm_100's FADD2/FMUL2/FFMA2 issue one instruction for both lanes).
//
// Per plane pair, the stage input (5 conserved components and the energy's
// low word) arrives in shared memory by two cp.async.bulk.tensor loads of
// the ghost-padded block: a box of 22 rows x the padded row x 2 planes, so
// the x and y halos are the block's own ghost zones.  The previous stage's
// epilogue keeps those current (it writes every cell it updates into the
// face ghosts that hold it, periodic, outflow or reflect as Parthenon's
// boundary exchange would).  Loads run one pair ahead on an mbarrier per
// slot; the staging costs no per-cell address arithmetic.
//
// Per pair the CTA then
//   1. converts the pair to primitives (rho, v, P, e_int; e_int = E - e_kin in
//      FP64 from the hi/lo energy) into an interleaved float2 buffer, the
//      thread's own column straight into its z window in registers;
//   2. x and y sweeps: reconstruction of every (primitive, cell) into shared
//      memory, then the Riemann flux of every face, then the divergence of the
//      thread's own two cells, accumulated in registers;
//   3. the z sweep in registers: reconstruction of the column's cells
//      (2j, 2j+1) from a six-plane window, the Riemann flux at faces
//      2j - 1/2 and 2j + 1/2;
//   4. the low-storage RK update of cells (2j - 1, 2j), the ghost copies of
//      the new state, and on the last stage the CFL estimate.
//
// The bulk modulus of the ideal gas is gamma P in every cell, and the
// reconstructions are homogeneous of degree one (WENO-Z's eps aside), so the
// face bulk modulus is gamma times the face pressure and six variables are
// reconstructed instead of the reference's seven (hydro_types.hpp:61-77).
//
// Arithmetic follows the reference expressions (reconstruction.hpp:11-142,
// riemann_solver.hpp:15-149, primconsflux.hpp:55-138, grid_update.hpp:15-57,
// grid.cpp:213-283, hydro_time_step.cpp:19-64) in FP32, with the
// rearrangements documented at each function; the FP32 path is checked
// against FP64 by its density L1 error.
#pragma once

#include <cuda.h>

#include <cfloat>
#include <cstdint>

#include "kmy_internal.hpp"

namespace kmy {
namespace slab {

constexpr int NX = 32;            // interior cells along x (one warp per row)
constexpr int TY = 16;            // rows per tile
constexpr int NT = NX * TY;       // threads per CTA, one column each
constexpr int HH = 3;             // staged halo cells on each side
constexpr int PC = NX + 2 * HH;   // 38 staged columns
constexpr int PR = TY + 2 * HH;   // 22 staged rows
constexpr int NV = 6;             // reconstructed: rho, v0, v1, v2, P, e_int
constexpr int NCV = 5;            // conserved components
enum : int { SD = 0, SV0 = 1, SPRES = 4, SEINT = 5 };

// x sweep: reconstruction cells -1 .. 32 (34) per row, 33 faces per row;
// y sweep: cells -1 .. 16 (18) per column, 17 faces per column.
constexpr int RXC = NX + 2, RYC = TY + 2;
constexpr int REC_N = (RXC * TY > RYC * NX ? RXC * TY : RYC * NX);  // 576 float2 per variable and side
constexpr int FX_N = (NX + 1) * TY, FY_N = NX * (TY + 1);
constexpr int FLX_N = FX_N > FY_N ? FX_N : FY_N;                    // 544 float2 per component

struct Args {
  MeshDesc m;
  float gm1, gam;
  int limiter;
  const float *u0;   // stage input (its interior cells feed the update)
  const float *u0lo;
  const float *ub;   // "base" container of the low-storage scheme
  const float *ublo;
  float *u1;         // stage output (interior and face ghosts)
  float *u1lo;
  int last;          // last stage: CFL estimate into the device clock
  double beta;
  DevClock *clock;
  int rgroup;        // padded rows per TMA row group (row stride x rgroup is a multiple of 16 bytes)
  int nty;           // tiles per block along y
  int nitems;        // blocks x tiles
};

// Shared-memory plan (bytes), the same on host and device.
struct Smem {
  int np0;
  __host__ __device__ explicit Smem(int np0_) : np0(np0_) {}
  __host__ __device__ static constexpr int rup(int x) { return (x + 127) & ~127; }
  __host__ __device__ int raw_plane() const { return PR * np0; }              // floats
  __host__ __device__ int raw_var() const { return 2 * raw_plane(); }         // floats
  __host__ __device__ int cc_bytes() const { return NCV * raw_var() * 4; }
  __host__ __device__ int lo_off() const { return rup(cc_bytes()); }
  __host__ __device__ int lo_bytes() const { return raw_var() * 4; }
  __host__ __device__ int slot_bytes() const { return rup(lo_off() + lo_bytes()); }
  __host__ __device__ int prim_off() const { return 2 * slot_bytes(); }
  __host__ __device__ static constexpr int prim_bytes() { return NV * PR * PC * 8; }
  __host__ __device__ int rec_off() const { return prim_off() + prim_bytes(); }
  __host__ __device__ static constexpr int rec_bytes() { return 2 * NV * REC_N * 8; }
  __host__ __device__ int flx_off() const { return rec_off() + rec_bytes(); }
  __host__ __device__ static constexpr int flx_bytes() { return NCV * FLX_N * 8; }
  __host__ __device__ int bar_off() const { return flx_off() + flx_bytes(); }
  __host__ __device__ int total() const { return bar_off() + 256; }
  // bytes one plane pair brings in (both tensor loads)
  __host__ __device__ int tx_bytes() const { return cc_bytes() + lo_bytes(); }
};

// ---------------------------------------------------------------------------
// TMA and mbarrier primitives (PTX ISA 8.x, sm_90 and later).
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
// Bounded wait for the phase of the given parity: false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < (1 << 22); it++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// Packed FP32 helpers.
__device__ __forceinline__ float2 psub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
// 2^(127 - E) for the biased exponent E of x >= 0: x times it lies in [1, 2).
__device__ __forceinline__ float exp_scale(float x) {
  return __uint_as_float(0x7f000000u - (__float_as_uint(x) & 0x7f800000u));
}

// WENO-Z at both faces of two cells (reconstruction.hpp:94-141), rearranged
// for FP32:
//  * the candidates enter as e1 + sum_k w_k (e_k - e1) with the differences
//    e0 - e1 and e2 - e1 written through the second differences u_k of the
//    smoothness indicators (one subtraction each instead of a 3-term stencil);
//  * the indicators are scaled by 12/13 (u^2 + (3/13) v^2), which leaves the
//    ratios tau / beta_k unchanged, and then by the power of two that puts the
//    largest into [1, 2);
//  * the reference's eps = 1e-36 becomes a floor of 1e-12 on the scaled
//    indicators: below it a stencil's weight already dominates by more than
//    1e24 and the FP32 sum no longer changes.  With the floor the product of
//    the three lies in [1e-36, 8], so one reciprocal gives all three ratios;
//    the two normalisations take one reciprocal each.
__device__ __forceinline__ void WenoZPair(const float2 (&s)[5], float2 &vM, float2 &vP) {
  const float2 a = s[0], b = s[1], c = s[2], d = s[3], e = s[4];
  const float2 m2 = p2(-2.f), m4 = p2(-4.f);
  const float2 u0 = pfma(m2, b, padd(a, c));
  const float2 u1 = pfma(m2, c, padd(b, d));
  const float2 u2 = pfma(m2, d, padd(c, e));
  const float2 c3 = pmul(p2(3.f), c);
  const float2 v0 = pfma(m4, b, padd(a, c3));
  const float2 v1 = psub2(b, d);
  const float2 v2 = pfma(m4, d, padd(e, c3));
  const float2 k = p2(3.f / 13.f);
  float2 b0 = pfma(u0, u0, pmul(pmul(k, v0), v0));
  float2 b1 = pfma(u1, u1, pmul(pmul(k, v1), v1));
  float2 b2 = pfma(u2, u2, pmul(pmul(k, v2), v2));
  const float2 sc = make_float2(exp_scale(fmaxf(b0.x, fmaxf(b1.x, b2.x))), exp_scale(fmaxf(b0.y, fmaxf(b1.y, b2.y))));
  b0 = pmul(b0, sc);
  b1 = pmul(b1, sc);
  b2 = pmul(b2, sc);
  const float2 ts = psub2(b2, b0);
  const float fl = 1.e-12f;
  const float2 D0 = make_float2(fmaxf(b0.x, fl), fmaxf(b0.y, fl));
  const float2 D1 = make_float2(fmaxf(b1.x, fl), fmaxf(b1.y, fl));
  const float2 D2 = make_float2(fmaxf(b2.x, fl), fmaxf(b2.y, fl));
  const float2 D01 = pmul(D0, D1);
  const float2 tR = pmul(ts, prcp(pmul(D01, D2)));
  const float2 r0 = pmul(tR, pmul(D1, D2)), r1 = pmul(tR, pmul(D0, D2)), r2 = pmul(tR, D01);
  const float2 one = p2(1.f);
  const float2 q0 = pfma(r0, r0, one), q1 = pfma(r1, r1, one), q2 = pfma(r2, r2, one);
  const float2 g0 = psub2(u0, u1), g2 = psub2(u2, u1);
  const float2 inner = pfma(p2(1.f / 12.f), u1, c);
  const float2 ep1 = pfma(p2(-0.25f), v1, inner), em1 = pfma(p2(0.25f), v1, inner);
  const float2 A = pmul(q0, g0), B = pmul(q2, g2);
  const float2 third = p2(1.f / 3.f), mhalf = p2(-0.5f);
  const float2 nP = pfma(A, third, pmul(mhalf, B));
  const float2 nM = pfma(B, third, pmul(mhalf, A));
  const float2 six = p2(6.f), three = p2(3.f);
  const float2 DP = pfma(three, q2, pfma(six, q1, q0));
  const float2 DM = pfma(three, q0, pfma(six, q1, q2));
  vP = pfma(nP, prcp(DP), ep1);
  vM = pfma(nM, prcp(DM), em1);
}

template <int RECON>
__device__ __forceinline__ void ReconPair(int limiter, const float2 (&s)[5], float2 &vM, float2 &vP) {
  if constexpr (RECON == WENOZ) {
    WenoZPair(s, vM, vP);
  } else {
    float lo[5], hi[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
      lo[k] = s[k].x;
      hi[k] = s[k].y;
    }
    Reconstruct<RECON, float>(limiter, lo, vM.x, vP.x);
    Reconstruct<RECON, float>(limiter, hi, vM.y, vP.y);
  }
}

// Riemann flux at two faces (riemann_solver.hpp:20-57 HLL, :59-149 HLLC) from
// the six reconstructed primitives of each side, face normal DIR1.
// The fast speed is sqrt(gamma P / rho) = gamma P / sqrt(gamma P rho) (one
// reciprocal square root).  HLLC blends the two star fluxes by
// max(tiny, sign u*) and -min(-tiny, sign u*); one of the two factors is tiny,
// so the flux is the star flux of the side that sign(u*) selects (u* = -0
// selects the right side, as copysign does), and only that state is formed.
// Its density ratio U*_rho / U_rho is susi (S - u_n), the reference's
// expression with rho cancelled.
template <int RIEMANN, int DIR1>
__device__ __forceinline__ void SlabRiemann2(const float2 *vL, const float2 *vR, float gam, float2 *F) {
  constexpr int DIR2 = (DIR1 + 1) % 3, DIR3 = (DIR1 + 2) % 3;
  const float tiny = FLT_MIN;
  const float2 uL = vL[SV0 + DIR1], uR = vR[SV0 + DIR1];
  const float2 gPL = pmul(p2(gam), vL[SPRES]), gPR = pmul(p2(gam), vR[SPRES]);
  const float2 tL = pmul(gPL, vL[SD]), tR = pmul(gPR, vR[SD]);
  const float2 cfL = pmul(gPL, make_float2(rsqrt_approx(fmaxf(tL.x, tiny)), rsqrt_approx(fmaxf(tL.y, tiny))));
  const float2 cfR = pmul(gPR, make_float2(rsqrt_approx(fmaxf(tR.x, tiny)), rsqrt_approx(fmaxf(tR.y, tiny))));
  const float2 mL = psub2(uL, cfL), mR = psub2(uR, cfR), pL = padd(uL, cfL), pR = padd(uR, cfR);
  const float2 sL = make_float2(fminf(-tiny, fminf(mL.x, mR.x)), fminf(-tiny, fminf(mL.y, mR.y)));
  const float2 sR = make_float2(fmaxf(tiny, fmaxf(pL.x, pR.x)), fmaxf(tiny, fmaxf(pL.y, pR.y)));
  if constexpr (RIEMANN == HLL) {
    // conserved state and flux of both sides (primconsflux.hpp:55-138)
    float2 UL[5], UR[5], FL[5], FR[5];
    auto cons_flux = [&](const float2 *V, float2 *U, float2 *Fx) {
      const float2 rho = V[SD], un = V[SV0 + DIR1];
      U[CDENS] = rho;
      Fx[CDENS] = pmul(rho, un);
#pragma unroll
      for (int dd = 0; dd < 3; dd++) {
        U[CMOM0 + dd] = pmul(rho, V[SV0 + dd]);
        Fx[CMOM0 + dd] = pmul(Fx[CDENS], V[SV0 + dd]);
      }
      const float2 vv = pfma(V[SV0 + 2], V[SV0 + 2], pfma(V[SV0 + 1], V[SV0 + 1], pmul(V[SV0], V[SV0])));
      U[CENER] = pfma(pmul(p2(0.5f), rho), vv, pmul(V[SEINT], rho));
      Fx[CMOM0 + DIR1] = padd(Fx[CMOM0 + DIR1], V[SPRES]);
      Fx[CENER] = pmul(padd(U[CENER], V[SPRES]), un);
    };
    cons_flux(vL, UL, FL);
    cons_flux(vR, UR, FR);
    const float2 sRmsLi = prcp(psub2(sR, sL)), sRsL = pmul(sR, sL);
#pragma unroll
    for (int v = 0; v < 5; v++)
      F[v] = pmul(sRmsLi, pfma(sRsL, psub2(UR[v], UL[v]), psub2(pmul(sR, FL[v]), pmul(sL, FR[v]))));
  } else {
    const float2 dL = psub2(sL, uL), dRn = psub2(uR, sR);  // dRn = -(sR - uR)
    const float2 rdL = pmul(vL[SD], dL), rdRn = pmul(vR[SD], dRn);
    // u* = (pR - pL + rhoL uL (sL - uL) - rhoR uR (sR - uR)) / (rhoL (sL - uL) - rhoR (sR - uR))
    const float2 num = pfma(rdRn, uR, pfma(rdL, uL, psub2(vR[SPRES], vL[SPRES])));
    const float2 ustar = pmul(num, prcp(padd(rdL, rdRn)));
    // p* = 0.5 (pL + pR + rhoL (sL - uL)(u* - uL) + rhoR (sR - uR)(u* - uR))
    const float2 pstar = pmul(p2(0.5f), pfma(rdRn, psub2(uR, ustar), pfma(rdL, psub2(ustar, uL), padd(vL[SPRES], vR[SPRES]))));
    // the side sign(u*) selects, per lane
    float2 S, rho, un, ut1, ut2, pr, ei;
    auto pick = [](float2 l, float2 r, bool xl, bool yl) { return make_float2(xl ? l.x : r.x, yl ? l.y : r.y); };
    const bool xl = !(__float_as_uint(ustar.x) >> 31), yl = !(__float_as_uint(ustar.y) >> 31);
    S = pick(sL, sR, xl, yl);
    rho = pick(vL[SD], vR[SD], xl, yl);
    un = pick(uL, uR, xl, yl);
    ut1 = pick(vL[SV0 + DIR2], vR[SV0 + DIR2], xl, yl);
    ut2 = pick(vL[SV0 + DIR3], vR[SV0 + DIR3], xl, yl);
    pr = pick(vL[SPRES], vR[SPRES], xl, yl);
    ei = pick(vL[SEINT], vR[SEINT], xl, yl);
    // U and F of that side along DIR1 (primconsflux.hpp:55-138)
    const float2 mn = pmul(rho, un), mt1 = pmul(rho, ut1), mt2 = pmul(rho, ut2);
    const float2 vv = pfma(ut2, ut2, pfma(ut1, ut1, pmul(un, un)));
    const float2 E = pfma(pmul(p2(0.5f), rho), vv, pmul(ei, rho));
    const float2 Fmn = pfma(mn, un, pr), Fmt1 = pmul(mn, ut1), Fmt2 = pmul(mn, ut2);
    const float2 FE = pmul(padd(E, pr), un);
    const float2 susi = prcp(padd(psub2(S, ustar), p2(tiny)));
    const float2 ratio = pmul(susi, psub2(S, un));
    const float2 Usr = pmul(rho, ratio);
    const float2 Usmn = pmul(Usr, ustar);
    const float2 Usmt1 = pmul(mt1, ratio), Usmt2 = pmul(mt2, ratio);
    const float2 UsE = pfma(E, ratio, pmul(susi, pfma(pstar, ustar, pmul(p2(-1.f), pmul(pr, un)))));
    F[CDENS] = pfma(S, psub2(Usr, rho), mn);
    F[CMOM0 + DIR1] = pfma(S, psub2(Usmn, mn), Fmn);
    F[CMOM0 + DIR2] = pfma(S, psub2(Usmt1, mt1), Fmt1);
    F[CMOM0 + DIR3] = pfma(S, psub2(Usmt2, mt2), Fmt2);
    F[CENER] = pfma(S, psub2(UsE, E), FE);
  }
}

// Primitives of one cell from its FP32 conserved state and energy low word
// (primconsflux.hpp:76-98 with the ideal-gas EOS of equation_of_state.hpp:53-64):
// e_int = (E_hi + E_lo) - |m|^2 / (2 rho) in FP64, with 1/rho from the FP32
// reciprocal and one Newton-Raphson step.
__device__ __forceinline__ void slab_prim(float gm1, float rho, float m0, float m1, float m2, float ehi, float elo,
                                          float (&V)[NV]) {
  const float r0 = rcp_approx(rho);
  V[SD] = rho;
  V[SV0] = m0 * r0;
  V[SV0 + 1] = m1 * r0;
  V[SV0 + 2] = m2 * r0;
  const double dd = double(rho), r0d = double(r0);
  const double id = fma(r0d, fma(-dd, r0d, 1.0), r0d);
  const double msq = fma(double(m0), double(m0), fma(double(m1), double(m1), double(m2) * double(m2)));
  const double eint = (double(ehi) + double(elo)) - 0.5 * msq * id;
  const float sie = float(eint * id);
  V[SEINT] = sie;
  V[SPRES] = fmaxf(0.f, gm1 * rho * sie);
}

// ---------------------------------------------------------------------------
// Face ghosts of the new state.  An interior cell at local index l along axis
// d is the source of the ghost cells that Parthenon's boundary exchange would
// fill from it: the high ghosts of the block below it (l < g), the low ghosts
// of the block above (l >= n - g), wrapped across a periodic boundary, and at
// an outflow or reflecting boundary its own block's ghosts (zero gradient; a
// mirror with the normal momentum negated).  Only face ghosts (the other two
// coordinates interior) are written: the sweeps read nothing else.
struct GhostVal {
  float v[NCV];
  float lo;
};

__device__ __forceinline__ void ghost_store(const Args &a, long long idx, const GhostVal &gv, int flip_d) {
  const long long NP = (long long)a.m.nb * a.m.P;
#pragma unroll
  for (int v = 0; v < NCV; v++) a.u1[v * NP + idx] = (v == CMOM0 + flip_d) ? -gv.v[v] : gv.v[v];
  a.u1lo[idx] = gv.lo;
}

__device__ __forceinline__ void ghost_push_axis(const Args &a, int d, int b, const int lb[3], const int pc[3],
                                                const GhostVal &gv) {
  const MeshDesc &m = a.m;
  const int n = m.nx[d], g = m.g[d], nbd = m.nbx[d];
  const int l = pc[d] - g;
  const long long stride = d == 0 ? 1 : d == 1 ? m.nbx[0] : (long long)m.nbx[0] * m.nbx[1];
  const long long sd = d == 0 ? 1 : d == 1 ? m.np[0] : (long long)m.np[0] * m.np[1];
  // element offset of (pc with coordinate d replaced by p) in block tb
  auto at = [&](long long tb, int p) {
    return tb * m.P + (long long)(pc[2] + (d == 2 ? p - pc[2] : 0)) * m.np[0] * m.np[1] +
           (long long)(pc[1] + (d == 1 ? p - pc[1] : 0)) * m.np[0] + (pc[0] + (d == 0 ? p - pc[0] : 0));
  };
  (void)sd;
  if (l < g) {
    if (lb[d] > 0 || m.bc[d][0] == BC_PERIODIC) {
      const long long tb = b + (lb[d] > 0 ? -stride : (long long)(nbd - 1) * stride);
      ghost_store(a, at(tb, n + g + l), gv, -9);
    } else if (m.bc[d][0] == BC_OUTFLOW) {
      if (l == 0)
        for (int p = 0; p < g; p++) ghost_store(a, at(b, p), gv, -9);
    } else {
      ghost_store(a, at(b, g - 1 - l), gv, d);
    }
  }
  if (l >= n - g) {
    if (lb[d] < nbd - 1 || m.bc[d][1] == BC_PERIODIC) {
      const long long tb = b + (lb[d] < nbd - 1 ? stride : -(long long)(nbd - 1) * stride);
      ghost_store(a, at(tb, l - n + g), gv, -9);
    } else if (m.bc[d][1] == BC_OUTFLOW) {
      if (l == n - 1)
        for (int p = 0; p < g; p++) ghost_store(a, at(b, n + g + p), gv, -9);
    } else {
      ghost_store(a, at(b, g + 2 * n - 1 - l), gv, d);
    }
  }
}

// ---------------------------------------------------------------------------
template <int RECON, int RIEMANN>
__global__ void __launch_bounds__(NT, 1)
    k_slab_stage(const __grid_constant__ CUtensorMap tm_cc, const __grid_constant__ CUtensorMap tm_lo,
                 const __grid_constant__ Args a) {
  extern __shared__ __align__(128) unsigned char smem[];
  const MeshDesc &m = a.m;
  const Smem L(m.np[0]);
  const int tid = threadIdx.x, lane = tid & 31, wr = tid >> 5;
  const int np0 = m.np[0], gx = m.g[0], nz = m.nx[2], nz2 = nz / 2;
  // raw slot s (s = pair & 1): the conserved box, then the energy low words
  auto raw = [&](int s) { return reinterpret_cast<float *>(smem + s * L.slot_bytes()); };
  auto rawlo = [&](int s) { return reinterpret_cast<float *>(smem + s * L.slot_bytes() + L.lo_off()); };
  float2 *prim = reinterpret_cast<float2 *>(smem + L.prim_off());   // [NV][PR][PC]
  float2 *rm = reinterpret_cast<float2 *>(smem + L.rec_off());      // [NV][REC_N]
  float2 *rp = rm + NV * REC_N;
  float2 *flx = reinterpret_cast<float2 *>(smem + L.flx_off());     // [NCV][FLX_N]
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L.bar_off());
  int *flag = reinterpret_cast<int *>(smem + L.bar_off() + 16);
  double *wmin = reinterpret_cast<double *>(smem + L.bar_off() + 64);

  const bool done = a.clock->done != 0;
  const double dt = a.clock->dt;
  const long long NP = (long long)m.nb * m.P;
  const float A0 = float(m.area[0]), A1 = float(m.area[1]), A2 = float(m.area[2]);
  const float vol = float(m.vol);
  const float bt = float(a.beta);
  const int RV = L.raw_var(), RPL = L.raw_plane();

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0u;  // bit s: parity of slot s's next completion
  double dtl = INFINITY;
  bool failed = false;

  for (int item = blockIdx.x; item < a.nitems && !failed; item += gridDim.x) {
    const int b = item / a.nty, ty = item - b * a.nty;
    const int oy = ty * TY;
    const int lb[3] = {b % m.nbx[0], (b / m.nbx[0]) % m.nbx[1], b / (m.nbx[0] * m.nbx[1])};
    const int row0 = oy + m.g[1] - HH;  // first staged padded row
    const int zc0 = b * m.np[2] + m.g[2];  // tensor plane coordinate of interior plane 0
    // this thread's column: interior (x, y) = (lane, oy + wr)
    const long long col = (long long)b * m.P + (long long)(oy + wr + m.g[1]) * np0 + (lane + gx);
    const long long plane_st = (long long)np0 * m.np[1];

    if (done) {
      // a stage queued after the run reached tlim leaves the state as it is
      for (int z = 0; z < nz; z++) {
        const long long n = col + (long long)(z + m.g[2]) * plane_st;
        GhostVal gv;
#pragma unroll
        for (int v = 0; v < NCV; v++) gv.v[v] = a.u0[v * NP + n];
        gv.lo = a.u0lo[n];
        if (a.u1 != a.u0) {
#pragma unroll
          for (int v = 0; v < NCV; v++) a.u1[v * NP + n] = gv.v[v];
          a.u1lo[n] = gv.lo;
        }
        const int pc[3] = {lane + gx, oy + wr + m.g[1], z + m.g[2]};
#pragma unroll
        for (int d = 0; d < 3; d++) ghost_push_axis(a, d, b, lb, pc, gv);
      }
      continue;
    }

    auto issue = [&](int pair) {
      if (tid == 0) {
        const int s = pair & 1;
        fence_proxy_async();
        mbar_expect_tx(&bar[s], unsigned(L.tx_bytes()));
        tma_load_4d(raw(s), &tm_cc, 0, row0 / a.rgroup, zc0 + 2 * pair, 0, &bar[s]);
        tma_load_3d(rawlo(s), &tm_lo, 0, row0 / a.rgroup, zc0 + 2 * pair, &bar[s]);
      }
    };
    // wait for a pair: thread 0 waits (bounded) and the CTA learns the outcome at the barrier
    auto wait_pair = [&](int pair) -> bool {
      const int s = pair & 1;
      const unsigned par = (phase >> s) & 1u;
      phase ^= 1u << s;
      if (tid == 0) *flag = mbar_wait(&bar[s], par) ? 0 : 1;
      __syncthreads();
      if (*flag) return false;
      mbar_wait(&bar[s], par);  // completes at once: the phase has flipped
      return true;
    };
    // own column of a pair -> primitives (float2 over the two planes)
    auto convert_own = [&](int pair, float2 (&W)[NV], bool keep) {
      const float *r = raw(pair & 1), *rl = rawlo(pair & 1);
      const int o = (wr + HH) * np0 + lane + gx;
      float V0[NV], V1[NV];
      slab_prim(a.gm1, r[o], r[RV + o], r[2 * RV + o], r[3 * RV + o], r[4 * RV + o], rl[o], V0);
      slab_prim(a.gm1, r[RPL + o], r[RV + RPL + o], r[2 * RV + RPL + o], r[3 * RV + RPL + o], r[4 * RV + RPL + o],
                rl[RPL + o], V1);
#pragma unroll
      for (int v = 0; v < NV; v++) W[v] = make_float2(V0[v], V1[v]);
      if (keep) {
#pragma unroll
        for (int v = 0; v < NV; v++) prim[(v * PR + wr + HH) * PC + lane + HH] = W[v];
      }
    };
    // the x and y halo cells of a centre pair
    auto convert_halo = [&](int pair) {
      const float *r = raw(pair & 1), *rl = rawlo(pair & 1);
      if (tid < 6 * TY + 6 * NX) {
        int rr, cc;
        if (tid < 6 * TY) {
          rr = HH + tid / 6;
          const int q = tid % 6;
          cc = q < 3 ? q : NX + q;
        } else {
          const int h = tid - 6 * TY;
          const int q = h / NX;
          rr = q < 3 ? q : TY + q;
          cc = HH + h % NX;
        }
        const int o = rr * np0 + cc - HH + gx;
        float V0[NV], V1[NV];
        slab_prim(a.gm1, r[o], r[RV + o], r[2 * RV + o], r[3 * RV + o], r[4 * RV + o], rl[o], V0);
        slab_prim(a.gm1, r[RPL + o], r[RV + RPL + o], r[2 * RV + RPL + o], r[3 * RV + RPL + o],
                  r[4 * RV + RPL + o], rl[RPL + o], V1);
#pragma unroll
        for (int v = 0; v < NV; v++) prim[(v * PR + rr) * PC + cc] = make_float2(V0[v], V1[v]);
      }
    };

    // the z window: planes (2j-2, 2j-1), (2j, 2j+1); carried z-face state
    float2 W0[NV], W1[NV], W2[NV];
    float vPc[NV], Fc[NCV], duc[NCV];
#pragma unroll
    for (int v = 0; v < NV; v++) vPc[v] = 0.f;
#pragma unroll
    for (int v = 0; v < NCV; v++) Fc[v] = duc[v] = 0.f;

    issue(-2);
    issue(-1);
    if (!wait_pair(-2)) {
      failed = true;
      break;
    }
    convert_own(-2, W0, false);
    __syncthreads();
    issue(0);
    if (!wait_pair(-1)) {
      failed = true;
      break;
    }
    convert_own(-1, W1, false);
    __syncthreads();

    for (int j = -1; j <= nz2; j++) {
      if (j + 2 <= nz2 + 1) issue(j + 2);
      // L2 prefetch of the rows this step's update reads
      {
        const int z0 = 2 * j - 1;
        if (lane < 24 && z0 + 1 >= 0 && z0 < nz) {
          const int arr = lane % 12, pl = lane / 12;
          const int z = z0 + pl;
          if (z >= 0 && z < nz) {
            const float *base = arr < 5 ? a.ub + arr * NP : arr == 5 ? a.ublo : arr < 11 ? a.u0 + (arr - 6) * NP : a.u0lo;
            const float *p = base + (long long)b * m.P + (long long)(z + m.g[2]) * plane_st +
                             (long long)(oy + wr + m.g[1]) * np0;
            const uintptr_t lo = uintptr_t(p) & ~uintptr_t(15);
            const unsigned bytes = unsigned(((uintptr_t(p + np0) & ~uintptr_t(15)) - lo));
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"(bytes) : "memory");
          }
        }
      }
      float2 du[NCV];
#pragma unroll
      for (int v = 0; v < NCV; v++) du[v] = p2(0.f);

      if (j >= 0 && j < nz2) {
        // ---- x sweep ----
        auto recon_x = [&](int v, int r, int xx) {
          const float2 *c = prim + (v * PR + r + HH) * PC + xx;
          float2 s[5];
#pragma unroll
          for (int q = 0; q < 5; q++) s[q] = c[q];
          float2 vm, vp;
          ReconPair<RECON>(a.limiter, s, vm, vp);
          rm[v * REC_N + r * RXC + xx] = vm;
          rp[v * REC_N + r * RXC + xx] = vp;
        };
#pragma unroll 1
        for (int v = 0; v < NV; v++) recon_x(v, wr, lane);
        if (tid < NV * TY * 2) recon_x(tid >> 5, (tid & 31) >> 1, NX + (tid & 1));
        __syncthreads();
        auto riemann_x = [&](int r, int f) {
          float2 vL[NV], vR[NV];
#pragma unroll
          for (int v = 0; v < NV; v++) {
            vL[v] = rp[v * REC_N + r * RXC + f];
            vR[v] = rm[v * REC_N + r * RXC + f + 1];
          }
          float2 F[NCV];
          SlabRiemann2<RIEMANN, 0>(vL, vR, a.gam, F);
#pragma unroll
          for (int v = 0; v < NCV; v++) flx[v * FLX_N + r * (NX + 1) + f] = F[v];
        };
        riemann_x(wr, lane);
        if (tid < TY) riemann_x(tid, NX);
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NCV; v++) {
          const float2 lo = flx[v * FLX_N + wr * (NX + 1) + lane], hi = flx[v * FLX_N + wr * (NX + 1) + lane + 1];
          du[v] = psub2(du[v], psub2(pmul(p2(A0), hi), pmul(p2(A0), lo)));
        }
        // ---- y sweep ----
        auto recon_y = [&](int v, int yy, int x) {
          const float2 *c = prim + (v * PR + yy) * PC + x + HH;
          float2 s[5];
#pragma unroll
          for (int q = 0; q < 5; q++) s[q] = c[q * PC];
          float2 vm, vp;
          ReconPair<RECON>(a.limiter, s, vm, vp);
          rm[v * REC_N + yy * NX + x] = vm;
          rp[v * REC_N + yy * NX + x] = vp;
        };
#pragma unroll 1
        for (int v = 0; v < NV; v++) recon_y(v, wr, lane);
        if (tid < NV * 2 * NX) recon_y(tid >> 6, TY + ((tid >> 5) & 1), lane);
        __syncthreads();
        auto riemann_y = [&](int f, int x) {
          float2 vL[NV], vR[NV];
#pragma unroll
          for (int v = 0; v < NV; v++) {
            vL[v] = rp[v * REC_N + f * NX + x];
            vR[v] = rm[v * REC_N + (f + 1) * NX + x];
          }
          float2 F[NCV];
          SlabRiemann2<RIEMANN, 1>(vL, vR, a.gam, F);
#pragma unroll
          for (int v = 0; v < NCV; v++) flx[v * FLX_N + f * NX + x] = F[v];
        };
        riemann_y(wr, lane);
        if (tid < NX) riemann_y(TY, tid);
        __syncthreads();
#pragma unroll
        for (int v = 0; v < NCV; v++) {
          const float2 lo = flx[v * FLX_N + wr * NX + lane], hi = flx[v * FLX_N + (wr + 1) * NX + lane];
          du[v] = psub2(du[v], psub2(pmul(p2(A1), hi), pmul(p2(A1), lo)));
        }
      }

      // ---- next pair: convert (own column into the window, and the halo if it is a centre pair) ----
      if (!wait_pair(j + 1)) {
        failed = true;
        break;
      }
      const bool centre = j + 1 >= 0 && j + 1 < nz2;
      convert_own(j + 1, W2, centre);
      if (centre) convert_halo(j + 1);

      // ---- z sweep in registers: cells (2j, 2j+1), faces 2j - 1/2 and 2j + 1/2 ----
      float2 vm[NV], vp[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const float2 s[5] = {W0[v], make_float2(W0[v].y, W1[v].x), W1[v], make_float2(W1[v].y, W2[v].x), W2[v]};
        ReconPair<RECON>(a.limiter, s, vm[v], vp[v]);
      }
      float2 vL[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) vL[v] = make_float2(vPc[v], vp[v].x);
      float2 F[NCV];
      SlabRiemann2<RIEMANN, 2>(vL, vm, a.gam, F);

      // ---- update of cells 2j-1 (lane x) and 2j (lane y) ----
      {
        float2 dz[NCV];
#pragma unroll
        for (int v = 0; v < NCV; v++) {
          // z contributions: -A (F+ - F-), after x and y as the reference sums them
          const float dA = duc[v] - (A2 * F[v].x - A2 * Fc[v]);
          const float dB = du[v].x - (A2 * F[v].y - A2 * F[v].x);
          dz[v] = make_float2(dA, dB);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int z = 2 * j - 1 + h;
          if (z < 0 || z >= nz) continue;
          const long long n = col + (long long)(z + m.g[2]) * plane_st;
          float zb[NCV], z0[NCV];
#pragma unroll
          for (int v = 0; v < NCV; v++) {
            zb[v] = a.ub[v * NP + n];
            z0[v] = a.u0[v * NP + n];
          }
          const float zblo = a.ublo[n], z0lo = a.u0lo[n];
          GhostVal gv;
#pragma unroll
          for (int v = 0; v < NCV; v++) {
            const float dudt = (h == 0 ? dz[v].x : dz[v].y) / vol;
            if (v == CENER) {
              const double eb = double(zb[v]) + double(zblo), e0 = double(z0[v]) + double(z0lo);
              const double e1 = (a.beta * eb + (1.0 - a.beta) * e0) + a.beta * dt * double(dudt);
              gv.v[v] = float(e1);
              gv.lo = float(e1 - double(gv.v[v]));
            } else {
              gv.v[v] = (bt * zb[v] + (1.f - bt) * z0[v]) + bt * float(dt) * dudt;
            }
            a.u1[v * NP + n] = gv.v[v];
          }
          a.u1lo[n] = gv.lo;
          const int pc[3] = {lane + gx, oy + wr + m.g[1], z + m.g[2]};
#pragma unroll
          for (int d = 0; d < 3; d++) ghost_push_axis(a, d, b, lb, pc, gv);
          if (a.last) {
            float V[NV];
            slab_prim(a.gm1, gv.v[0], gv.v[1], gv.v[2], gv.v[3], gv.v[4], gv.lo, V);
#pragma unroll
            for (int d = 0; d < 3; d++) {
              const float cf = sqrtf(a.gam * V[SPRES] / V[SD]);
              double xv = double(float(m.dx[d]) / (fabsf(V[SV0 + d]) + cf));
              if (xv != xv) xv = 0.0;
              dtl = xv < dtl ? xv : dtl;
            }
          }
        }
      }
      // carry to the next pair
#pragma unroll
      for (int v = 0; v < NV; v++) {
        vPc[v] = vp[v].y;
        W0[v] = W1[v];
        W1[v] = W2[v];
      }
#pragma unroll
      for (int v = 0; v < NCV; v++) {
        Fc[v] = F[v].y;
        duc[v] = du[v].y;
      }
      __syncthreads();
    }
  }
  if (failed) {
    if (tid == 0) atomicExch(&a.clock->status, int(KMY_ERR_TIMEOUT));
    return;
  }
  if (a.last && !done) {
    for (int q = 16; q > 0; q >>= 1) dtl = fmin(dtl, __shfl_xor_sync(0xffffffffu, dtl, q));
    if (lane == 0) wmin[wr] = dtl;
    __syncthreads();
    if (tid == 0) {
      double v = wmin[0];
      for (int w = 1; w < NT / 32; w++) v = fmin(v, wmin[w]);
      if (!(v >= 0.0)) v = 0.0;
      if (v < INFINITY) atomicMin(&a.clock->dtmin_bits, (unsigned long long)__double_as_longlong(v));
    }
  }
}

}  // namespace slab
}  // namespace kmy

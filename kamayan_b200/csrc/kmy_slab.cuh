// kmy_slab.cuh -- one RK stage of 3D hydro, streamed through each meshblock
// along z with TMA-staged plane pairs, in FP32 or FP64.
//
// Work item: one meshblock b and one tile of TY rows (y) by the block's full
// 32-cell width (x).  A persistent grid strides over the (block, tile) work
// list: in FP32, TY = 16 runs one CTA of 512 threads per SM, TY = 8 two CTAs
// of 256 (they fill each other's barrier waits; the staged halo rows cost
// more); in FP64 (twice the shared memory per cell) TY = 8 runs one CTA of
// 256 per SM.  Thread t owns the column (x = t % 32, y = oy + t / 32) and
// walks it along z two planes at a time: every operation of the z sweep works
// on a pair of planes (k, k+1).  In FP32 the pair is a float2 and sm_100's
// FADD2/FMUL2/FFMA2 issue one instruction for both lanes; in FP64 it is a
// double2 worked lane by lane (two independent dependency chains per thread).
//
// Per plane pair, the stage input (5 conserved components, and in FP32 the
// energy's low word) arrives in shared memory by cp.async.bulk.tensor loads
// of the ghost-padded block: a box of TY + 6 rows x the padded row x 2
// planes, so the x and y halos are the block's own ghost zones.  The previous
// stage's epilogue keeps those current (it writes every cell it updates into
// the face ghosts that hold it, periodic, outflow or reflect as Parthenon's
// boundary exchange would).  The loads of the next pair are issued as soon as
// the raw slot is converted and land while the CTA works on the current pair
// (one mbarrier, bounded waits); the staging costs no per-cell address
// arithmetic.
//
// Per pair the CTA then
//   1. converts the pair to primitives (rho, v, P, e_int; in FP32 e_int =
//      E - e_kin in FP64 from the hi/lo energy) into an interleaved pair
//      buffer, the thread's own column straight into its z window in registers;
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
// grid.cpp:213-283, hydro_time_step.cpp:19-64).  FP64 calls the per-cell
// device functions of the other FP64 stages (Reconstruct, WenoZBothTwoDiv,
// RiemannFlux, Cons2PrimEos) lane by lane and is checked against the oracle;
// FP32 uses the packed rearrangements documented at each function and is
// checked against FP64 by its density L1 error.
#pragma once

#include <cuda.h>

#include <cfloat>
#include <cstdint>

#include "kmy_internal.hpp"

// FP64 divisions and square roots of the z-streamed stage (reconstruction,
// conversion, HLLC) as Newton-Raphson refinements (rcp_nr, sqrt_nr) rather
// than IEEE division and square root; 0 builds the IEEE form.
#ifndef SLAB_F64_NR
#define SLAB_F64_NR 1
#endif
#ifndef SLAB_Y_EXTRAS_LAST_WARP
#define SLAB_Y_EXTRAS_LAST_WARP 1
#endif
// Unrolling of the constrained-transport stage's loops: the x and y
// reconstruction loops over the nine variables, and the two lanes of its
// per-lane MHD Riemann solver.
#ifndef SLAB_MHD_UNROLL
#define SLAB_MHD_UNROLL 1
#endif
#ifndef SLAB_MHD_LANES
#define SLAB_MHD_LANES 2
#endif

namespace kmy {

// Pair arithmetic on double2, lane by lane (the float2 forms are packed
// instructions, kmy_device.cuh).
__device__ __forceinline__ double2 padd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 pmul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }

namespace slab {

constexpr int NX = 32;            // interior cells along x (one warp per row)
constexpr int HH = 3;             // staged halo cells on each side
constexpr int PC = NX + 2 * HH;   // 38 staged columns
constexpr int NV = 6;             // reconstructed: rho, v0, v1, v2, P, e_int
constexpr int NCV = 5;            // conserved components the stage updates
enum : int { SD = 0, SV0 = 1, SPRES = 4, SEINT = 5, SB0 = 6 };
// With constrained transport the cell-centred field is reconstructed too
// (slots SB0 .. SB0 + 2) and staged with the other conserved components; the
// stage updates the five hydro components (the field is the faces' business).
template <bool MHD> struct Vars {
  static constexpr int NV = MHD ? 9 : 6;   // reconstructed
  static constexpr int NCC = MHD ? 8 : 5;  // staged conserved components
};

// Pair of two planes' values: packed FP32, or FP64 worked lane by lane.
template <typename R> struct PairOf;
template <> struct PairOf<float> { using T = float2; };
template <> struct PairOf<double> { using T = double2; };

// Tile of TY rows.  FP32: 16 (one CTA of 512 threads per SM) or 8 (two CTAs
// of 256); FP64: 8 (one CTA of 256).
// x sweep: reconstruction cells -1 .. 32 (34) per row, 33 faces per row;
// y sweep: cells -1 .. TY (TY + 2) per column, TY + 1 faces per column.
template <int TY_, typename R, bool MHD = false>
struct Tile {
  static constexpr int TY = TY_;
  static constexpr int NT = NX * TY;      // threads, one column each
  static constexpr int PR = TY + 2 * HH;  // staged rows
  static constexpr int CTAS = (TY == 8 && sizeof(R) == 4 && !MHD) ? 2 : 1;  // CTAs per SM the plan is sized for
  static constexpr int RXC = NX + 2, RYC = TY + 2;
  static constexpr int REC_N = RXC * TY > RYC * NX ? RXC * TY : RYC * NX;  // pairs per variable and side
  static constexpr int FX_N = (NX + 1) * TY, FY_N = NX * (TY + 1);
  static constexpr int FLX_N = FX_N > FY_N ? FX_N : FY_N;                  // pairs per component
};

template <typename R>
struct Args {
  MeshDesc m;
  EosParams eos;     // the FP64 conversion (Cons2PrimEos)
  R gm1, gam;
  int limiter;
  const R *u0;       // stage input (its interior cells feed the update)
  const float *u0lo; // FP32: energy low words (null in FP64)
  const R *ub;       // "base" container of the low-storage scheme
  const float *ublo;
  R *u1;             // stage output (interior and face ghosts)
  float *u1lo;
  int last;          // last stage: CFL estimate into the device clock
  double beta;
  DevClock *clock;
  int rgroup;        // padded rows per TMA row group (row stride x rgroup is a multiple of 16 bytes)
  int nty;           // tiles per block along y
  int nitems;        // blocks x tiles
  // the staged-pair wait: iterations of mbarrier.try_wait before it gives up,
  // and extra bytes the barrier expects beyond what the loads deliver (0; a
  // test sets it, with a short limit, to make the wait run out)
  int wait_limit;
  unsigned tx_extra;
  // constrained transport: the stage input's face field (the Riemann
  // problems' normal component) and the face-flux arrays the edge EMFs read,
  // layout [dir][8][nb * Pf]
  const R *fc0;
  R *flux;
};

// Shared-memory plan (bytes), the same on host and device: one raw slot (the
// stage input of one plane pair as the tensor loads deliver it), the
// interleaved primitives of the centre pair, the reconstructed face values
// and the face fluxes of one sweep, the mbarrier and reduction scratch.
template <int TY, typename R, bool MHD = false>
struct Smem {
  using T = Tile<TY, R, MHD>;
  static constexpr int NVK = Vars<MHD>::NV, NCCK = Vars<MHD>::NCC;
  static constexpr int ES = int(sizeof(R));      // bytes per staged value
  static constexpr int PS = 2 * int(sizeof(R));  // bytes per pair
  static constexpr bool LO = sizeof(R) == 4;     // FP32 stages the energy low words too
  int np0;
  __host__ __device__ explicit Smem(int np0_) : np0(np0_) {}
  __host__ __device__ static constexpr int rup(int x) { return (x + 127) & ~127; }
  __host__ __device__ int raw_plane() const { return T::PR * np0; }           // values
  __host__ __device__ int raw_var() const { return 2 * raw_plane(); }         // values
  __host__ __device__ int cc_bytes() const { return NCCK * raw_var() * ES; }
  __host__ __device__ int lo_off() const { return rup(cc_bytes()); }
  __host__ __device__ int lo_bytes() const { return LO ? raw_var() * 4 : 0; }
  __host__ __device__ int slot_bytes() const { return rup(lo_off() + lo_bytes()); }
  __host__ __device__ int prim_off() const { return slot_bytes(); }
  __host__ __device__ static constexpr int prim_bytes() { return NVK * T::PR * PC * PS; }
  __host__ __device__ int rec_off() const { return prim_off() + prim_bytes(); }
  __host__ __device__ static constexpr int rec_bytes() { return 2 * NVK * T::REC_N * PS; }
  __host__ __device__ int flx_off() const { return rec_off() + rec_bytes(); }
  __host__ __device__ static constexpr int flx_bytes() { return NCV * T::FLX_N * PS; }
  __host__ __device__ int bar_off() const { return flx_off() + flx_bytes(); }
  __host__ __device__ int total() const { return bar_off() + 256; }
  // bytes one plane pair brings in (all tensor loads)
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
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int limit) {
  const uint32_t a = smem_u32(bar);
  for (int it = 0; it < limit; it++) {
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
// Pair helpers.
// a - b; in FP32 one packed FMA, a + (-1) b
__device__ __forceinline__ float2 psub2(float2 a, float2 b) { return __ffma2_rn(make_float2(-1.f, -1.f), b, a); }
__device__ __forceinline__ double2 psub2(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk2(double a, double b) { return make_double2(a, b); }
template <typename R> __device__ __forceinline__ typename PairOf<R>::T splat(R a) { return mk2(a, a); }
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
//    ratios tau / (eps + beta_k) unchanged up to eps;
//  * each ratio takes one reciprocal and is capped at 1e15 so its square
//    stays finite in FP32: at that ratio the stencil already holds the whole
//    weight.  The clamps run on the ALU pipe, which the stage leaves mostly
//    idle; an eps scaled to the indicators (no clamps) cost five more
//    FMA-pipe operations per pair and measured slower.
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
  const float2 k = p2(3.f / 13.f), eps = p2(1.e-36f);
  const float2 D0 = pfma(u0, u0, pfma(pmul(k, v0), v0, eps));
  const float2 D1 = pfma(u1, u1, pfma(pmul(k, v1), v1, eps));
  const float2 D2 = pfma(u2, u2, pfma(pmul(k, v2), v2, eps));
  const float2 tau = psub2(D2, D0);
  const float cap = 1.e15f;
  const float2 r0 = pmul(tau, prcp(D0)), r1 = pmul(tau, prcp(D1)), r2 = pmul(tau, prcp(D2));
  const float2 r0c = make_float2(fminf(fabsf(r0.x), cap), fminf(fabsf(r0.y), cap));
  const float2 r1c = make_float2(fminf(fabsf(r1.x), cap), fminf(fabsf(r1.y), cap));
  const float2 r2c = make_float2(fminf(fabsf(r2.x), cap), fminf(fabsf(r2.y), cap));
  const float2 one = p2(1.f);
  const float2 q0 = pfma(r0c, r0c, one), q1 = pfma(r1c, r1c, one), q2 = pfma(r2c, r2c, one);
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

// FP64 division and square root: the Newton-Raphson forms (rcp_nr, sqrt_nr,
// DivNR in kmy_device.cuh) or IEEE.
#if SLAB_F64_NR
using SlabDiv64 = DivNR;
__device__ __forceinline__ double slab_sqrt64(double a) { return sqrt_nr(a); }
#else
using SlabDiv64 = DivIeee;
__device__ __forceinline__ double slab_sqrt64(double a) { return sqrt(a); }
#endif

// FP64: the per-cell reconstructions of the other FP64 stages, lane by lane
// (WENO-Z in its two-division form, the divisions as Newton-Raphson
// reciprocals).
template <int RECON>
__device__ __forceinline__ void ReconPair(int limiter, const double2 (&s)[5], double2 &vM, double2 &vP) {
  double lo[5], hi[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    lo[k] = s[k].x;
    hi[k] = s[k].y;
  }
  if constexpr (RECON == WENOZ) {
    WenoZBothTwoDiv<double, SlabDiv64>(lo, vM.x, vP.x);
    WenoZBothTwoDiv<double, SlabDiv64>(hi, vM.y, vP.y);
  } else {
    Reconstruct<RECON, double>(limiter, lo, vM.x, vP.x);
    Reconstruct<RECON, double>(limiter, hi, vM.y, vP.y);
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
  // (+ FLT_MIN keeps the reciprocal square root finite where P = 0)
  const float2 tLs = padd(tL, p2(tiny)), tRs = padd(tR, p2(tiny));
  const float2 cfL = pmul(gPL, make_float2(rsqrt_approx(tLs.x), rsqrt_approx(tLs.y)));
  const float2 cfR = pmul(gPR, make_float2(rsqrt_approx(tRs.x), rsqrt_approx(tRs.y)));
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

// FP64 HLLC at one face (riemann_solver.hpp:59-149) from the six
// reconstructed primitives of each side.  The reference blends the two star
// fluxes by max(tiny, sign u*) and -min(-tiny, sign u*); one factor is
// DBL_MIN, so the flux is the star flux of the side sign(u*) selects (u* = -0
// selects the right side, as copysign does) and only that state is formed.
// Its density ratio U*_rho / U_rho is susi (S - u_n), the reference's
// expression with rho cancelled (one division instead of two per side).
template <int DIR1>
__device__ __forceinline__ void hllc64(const double (&L)[NV], const double (&Rv)[NV], double gam, double *F) {
  constexpr int DIR2 = (DIR1 + 1) % 3, DIR3 = (DIR1 + 2) % 3;
  const double tiny = DBL_MIN;
  const double uL = L[SV0 + DIR1], uR = Rv[SV0 + DIR1];
  // FastSpeed: sqrt(bulk modulus / rho), bulk modulus gamma P
  const double cfL = slab_sqrt64(SlabDiv64::div(1.0, L[SD]) * (gam * L[SPRES]));
  const double cfR = slab_sqrt64(SlabDiv64::div(1.0, Rv[SD]) * (gam * Rv[SPRES]));
  const double sL = kmin(-tiny, kmin(uL - cfL, uR - cfR));
  const double sR = kmax(tiny, kmax(uL + cfL, uR + cfR));
  const double dL = sL - uL, dR = sR - uR;
  double ustar = Rv[SPRES] - L[SPRES] + (L[SD] * uL) * dL - (Rv[SD] * uR) * dR;
  ustar = SlabDiv64::div(ustar, L[SD] * dL - Rv[SD] * dR);
  const double pstar = 0.5 * (L[SPRES] + Rv[SPRES] + L[SD] * dL * (ustar - uL) + Rv[SD] * dR * (ustar - uR));
  const bool left = !signbit(ustar);
  const double S = left ? sL : sR;
  double V[NV];
#pragma unroll
  for (int v = 0; v < NV; v++) V[v] = left ? L[v] : Rv[v];
  const double rho = V[SD], un = V[SV0 + DIR1], pr = V[SPRES];
  // U and F of that side along DIR1 (primconsflux.hpp:55-138)
  const double mn = rho * un, mt1 = rho * V[SV0 + DIR2], mt2 = rho * V[SV0 + DIR3];
  double ekin = 0.0;
  ekin += V[SV0] * V[SV0];
  ekin += V[SV0 + 1] * V[SV0 + 1];
  ekin += V[SV0 + 2] * V[SV0 + 2];
  const double E = V[SEINT] * rho + ekin * (0.5 * rho);
  const double susi = SlabDiv64::div(1.0, S - ustar + tiny);
  const double Usr = susi * (S * rho - mn);
  const double ratio = susi * (S - un);
  F[CDENS] = mn + S * (Usr - rho);
  F[CMOM0 + DIR1] = (mn * un + pr) + S * (Usr * ustar - mn);
  F[CMOM0 + DIR2] = mn * V[SV0 + DIR2] + S * (mt1 * ratio - mt1);
  F[CMOM0 + DIR3] = mn * V[SV0 + DIR3] + S * (mt2 * ratio - mt2);
  F[CENER] = (E + pr) * un + S * ((E * ratio + susi * (pstar * ustar - pr * un)) - E);
}

// FP64 Riemann flux at two faces, lane by lane: HLLC as above, HLL through
// RiemannFlux (riemann_solver.hpp:20-57) with the face bulk modulus gamma P.
template <int RIEMANN, int DIR1>
__device__ __forceinline__ void SlabRiemann2(const double2 *vL, const double2 *vR, double gam, double2 *F) {
  double fl[2][NCV];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    auto lane = [h](double2 p) { return h ? p.y : p.x; };
    if constexpr (RIEMANN == HLLC) {
      double L[NV], Rv[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        L[v] = lane(vL[v]);
        Rv[v] = lane(vR[v]);
      }
      hllc64<DIR1>(L, Rv, gam, fl[h]);
    } else {
      double L[7], Rv[7];
      L[RDENS] = lane(vL[SD]);
      Rv[RDENS] = lane(vR[SD]);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        L[RVEL0 + d] = lane(vL[SV0 + d]);
        Rv[RVEL0 + d] = lane(vR[SV0 + d]);
      }
      L[RPRES] = lane(vL[SPRES]);
      Rv[RPRES] = lane(vR[SPRES]);
      L[RBMOD] = gam * L[RPRES];
      Rv[RBMOD] = gam * Rv[RPRES];
      L[REINT] = lane(vL[SEINT]);
      Rv[REINT] = lane(vR[SEINT]);
      RiemannFlux<RIEMANN, false, DIR1, double>(L, Rv, fl[h]);
    }
  }
#pragma unroll
  for (int v = 0; v < NCV; v++) F[v] = make_double2(fl[0][v], fl[1][v]);
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

// FP64: Cons2Prim with the ideal-gas EOS (primconsflux.hpp:76-98,
// equation_of_state.hpp:53-64) in Cons2PrimEos's order, 1/rho through the
// stage's reciprocal.
__device__ __forceinline__ void slab_prim(const EosParams &eos, double rho, double m0, double m1, double m2,
                                          double ener, double (&V)[NV]) {
  const double idens = SlabDiv64::div(1.0, rho);
  V[SD] = rho;
  V[SV0] = idens * m0;
  V[SV0 + 1] = idens * m1;
  V[SV0 + 2] = idens * m2;
  double ekin = 0.0;
  ekin += V[SV0] * V[SV0];
  ekin += V[SV0 + 1] * V[SV0 + 1];
  ekin += V[SV0 + 2] * V[SV0 + 2];
  ekin *= 0.5 * rho;
  const double sie = idens * (ener - ekin);
  V[SEINT] = sie;
  V[SPRES] = kmax(0.0, eos.gm1 * rho * sie);
}

// Constrained transport, FP32: the primitives of a staged cell with its
// cell-centred field; e_int = (E_hi + E_lo) - |m|^2 / (2 rho) - |B|^2 / 2 in
// FP64 (primconsflux.hpp:76-98).
__device__ __forceinline__ void slab_prim_mhd(float gm1, const float (&u)[8], float elo, float (&V)[9]) {
  const float rho = u[CDENS];
  const float r0 = rcp_approx(rho);
  V[SD] = rho;
#pragma unroll
  for (int d = 0; d < 3; d++) V[SV0 + d] = u[CMOM0 + d] * r0;
  const double dd = double(rho), r0d = double(r0);
  const double id = fma(r0d, fma(-dd, r0d, 1.0), r0d);
  const double msq = fma(double(u[CMOM0]), double(u[CMOM0]),
                         fma(double(u[CMOM1]), double(u[CMOM1]), double(u[CMOM2]) * double(u[CMOM2])));
  const double bsq = fma(double(u[CMAGC0]), double(u[CMAGC0]),
                         fma(double(u[CMAGC0 + 1]), double(u[CMAGC0 + 1]),
                             double(u[CMAGC0 + 2]) * double(u[CMAGC0 + 2])));
  const double eint = ((double(u[CENER]) + double(elo)) - 0.5 * msq * id) - 0.5 * bsq;
  const float sie = float(eint * id);
  V[SEINT] = sie;
  V[SPRES] = fmaxf(0.f, gm1 * rho * sie);
#pragma unroll
  for (int d = 0; d < 3; d++) V[SB0 + d] = u[CMAGC0 + d];
}

// Constrained transport, FP32: the MHD Riemann flux at two faces, lane by lane
// through RiemannFlux<RIEMANN, MHD> (riemann_solver.hpp:20-149), with the face
// field bn as the normal component of both states
// (hydro_add_flux_tasks.cpp:343-346) and the face bulk modulus gamma P.  F
// gets the five hydro fluxes; Bt[lane][0 / 1] the fluxes of the two
// transverse field components (DIR1 + 1, DIR1 + 2 mod 3 in increasing axis
// order), which the edge EMFs read.
template <int RIEMANN, int DIR1>
__device__ __forceinline__ void SlabRiemannMHD2(const float2 *vL, const float2 *vR, float gam, float2 bn,
                                                float2 *F, float (&Bt)[2][2]) {
  float fl[2][8];
  constexpr int LANES = SLAB_MHD_LANES;
#pragma unroll(LANES)
  for (int h = 0; h < 2; h++) {
    auto lane = [h](float2 p) { return h ? p.y : p.x; };
    float L[10], Rv[10];
    L[RDENS] = lane(vL[SD]);
    Rv[RDENS] = lane(vR[SD]);
#pragma unroll
    for (int d = 0; d < 3; d++) {
      L[RVEL0 + d] = lane(vL[SV0 + d]);
      Rv[RVEL0 + d] = lane(vR[SV0 + d]);
      L[RMAGC0 + d] = lane(vL[SB0 + d]);
      Rv[RMAGC0 + d] = lane(vR[SB0 + d]);
    }
    L[RPRES] = lane(vL[SPRES]);
    Rv[RPRES] = lane(vR[SPRES]);
    L[RBMOD] = gam * L[RPRES];
    Rv[RBMOD] = gam * Rv[RPRES];
    L[REINT] = lane(vL[SEINT]);
    Rv[REINT] = lane(vR[SEINT]);
    L[RMAGC0 + DIR1] = Rv[RMAGC0 + DIR1] = lane(bn);
    RiemannFlux<RIEMANN, true, DIR1, float>(L, Rv, fl[h]);
    constexpr int T0 = DIR1 == 0 ? 1 : 0, T1 = DIR1 == 2 ? 1 : 2;
    Bt[h][0] = fl[h][CMAGC0 + T0];
    Bt[h][1] = fl[h][CMAGC0 + T1];
  }
#pragma unroll
  for (int v = 0; v < NCV; v++) F[v] = make_float2(fl[0][v], fl[1][v]);
}

// ---------------------------------------------------------------------------
// Face ghosts of the new state.  An interior cell at local index l along axis
// d is the source of the ghost cells that Parthenon's boundary exchange would
// fill from it: the high ghosts of the block below it (l < g), the low ghosts
// of the block above (l >= n - g), wrapped across a periodic boundary, and at
// an outflow or reflecting boundary its own block's ghosts (zero gradient; a
// mirror with the normal momentum negated).  Only face ghosts (the other two
// coordinates interior) are written: the sweeps read nothing else.
template <typename R>
struct GhostVal {
  R v[NCV];
  float lo;  // FP32: the energy's low word
};

template <typename R>
__device__ __forceinline__ void ghost_store(const Args<R> &a, long long idx, const GhostVal<R> &gv, int flip_d) {
  const long long NP = (long long)a.m.nb * a.m.P;
#pragma unroll
  for (int v = 0; v < NCV; v++) a.u1[v * NP + idx] = (v == CMOM0 + flip_d) ? -gv.v[v] : gv.v[v];
  if constexpr (sizeof(R) == 4) a.u1lo[idx] = gv.lo;
}

template <typename R>
__device__ __forceinline__ void ghost_push_axis(const Args<R> &a, int d, int b, const int lb[3], const int pc[3],
                                                const GhostVal<R> &gv) {
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
#ifndef SLAB_F64_UNROLL
#define SLAB_F64_UNROLL 1
#endif


// The stage kernel.  tm_cc maps the stage input's conserved components;
// tm_lo its energy low words (FP32; unused in FP64).  MHD: constrained
// transport (FP32): nine reconstructed variables, the face field as the
// normal B of every Riemann problem, the transverse field fluxes written out.
template <typename R, int TY_, int RECON, int RIEMANN, bool MHD = false>
__global__ void __launch_bounds__(Tile<TY_, R, MHD>::NT, Tile<TY_, R, MHD>::CTAS)
    k_slab_stage(const __grid_constant__ CUtensorMap tm_cc, const __grid_constant__ CUtensorMap tm_lo,
                 const __grid_constant__ Args<R> a) {
  using T = Tile<TY_, R, MHD>;
  using P = typename PairOf<R>::T;
  constexpr bool LO = sizeof(R) == 4;
  static_assert(!MHD || LO, "the constrained-transport stage is FP32");
  constexpr int NV = Vars<MHD>::NV, NCC = Vars<MHD>::NCC;
  constexpr int TY = T::TY, NT = T::NT, PR = T::PR, RXC = T::RXC, REC_N = T::REC_N, FLX_N = T::FLX_N;
  // unrolling of the x and y reconstruction loops over the variables
  constexpr int RU = LO ? (MHD ? SLAB_MHD_UNROLL : NV) : SLAB_F64_UNROLL;
  extern __shared__ __align__(128) unsigned char smem[];
  const MeshDesc &m = a.m;
  const Smem<TY_, R, MHD> L(m.np[0]);
  const int tid = threadIdx.x, lane = tid & 31, wr = tid >> 5;
  const int np0 = m.np[0], gx = m.g[0], nz = m.nx[2], nz2 = nz / 2;
  // the raw slot: the conserved box of a plane pair, then (FP32) its energy low words
  R *const rawcc = reinterpret_cast<R *>(smem);
  float *const rawlo = reinterpret_cast<float *>(smem + L.lo_off());
  P *prim = reinterpret_cast<P *>(smem + L.prim_off());   // [NV][PR][PC]
  P *rm = reinterpret_cast<P *>(smem + L.rec_off());      // [NV][REC_N]
  P *rp = rm + NV * REC_N;
  P *flx = reinterpret_cast<P *>(smem + L.flx_off());     // [NCV][FLX_N]
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L.bar_off());
  int *flag = reinterpret_cast<int *>(smem + L.bar_off() + 16);
  double *wmin = reinterpret_cast<double *>(smem + L.bar_off() + 64);

  const bool done = a.clock->done != 0;
  const double dt = a.clock->dt;
  const long long NP = (long long)m.nb * m.P;
  const R A0 = R(m.area[0]), A1 = R(m.area[1]), A2 = R(m.area[2]);
  const R vol = R(m.vol);
  const R bt = R(a.beta);
  const int RV = L.raw_var(), RPL = L.raw_plane();
  const long long plane_st = (long long)np0 * m.np[1];

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned phase = 0u;  // parity of the slot's next completion
  double dtl = INFINITY;
  bool failed = false;

  for (int item = blockIdx.x; item < a.nitems && !failed; item += gridDim.x) {
    const int b = item / a.nty, ty = item - b * a.nty;
    const int oy = ty * TY;
    const int lb[3] = {b % m.nbx[0], (b / m.nbx[0]) % m.nbx[1], b / (m.nbx[0] * m.nbx[1])};
    const int row0 = oy + m.g[1] - HH;     // first staged padded row
    const int zc0 = b * m.np[2] + m.g[2];  // tensor plane coordinate of interior plane 0
    // this thread's column: interior (x, y) = (lane, oy + wr)
    const long long col = (long long)b * m.P + (long long)(oy + wr + m.g[1]) * np0 + (lane + gx);
    // whether the column lies within g of an x or y block face (its cells fill face ghosts)
    const bool px = lane < gx || lane >= NX - gx;
    const bool py = oy + wr < m.g[1] || oy + wr >= m.nx[1] - m.g[1];

    if (done) {
      // a stage queued after the run reached tlim leaves the state as it is
      for (int z = 0; z < nz; z++) {
        const long long n = col + (long long)(z + m.g[2]) * plane_st;
        GhostVal<R> gv;
#pragma unroll
        for (int v = 0; v < NCV; v++) gv.v[v] = a.u0[v * NP + n];
        gv.lo = LO ? a.u0lo[n] : 0.f;
        if (a.u1 != a.u0) {
#pragma unroll
          for (int v = 0; v < NCC; v++) a.u1[v * NP + n] = a.u0[v * NP + n];
          if constexpr (LO) a.u1lo[n] = gv.lo;
        }
        const int pc[3] = {lane + gx, oy + wr + m.g[1], z + m.g[2]};
#pragma unroll
        for (int d = 0; d < 3; d++) ghost_push_axis(a, d, b, lb, pc, gv);
      }
      continue;
    }

    // the tensor loads of a plane pair into the raw slot (free: the pair
    // before it was converted before the last barrier)
    auto issue = [&](int pair) {
      if (tid == 0) {
        fence_proxy_async();
        mbar_expect_tx(&bar[0], unsigned(L.tx_bytes()) + a.tx_extra);
        tma_load_4d(rawcc, &tm_cc, 0, row0 / a.rgroup, zc0 + 2 * pair, 0, &bar[0]);
        if constexpr (LO) tma_load_3d(rawlo, &tm_lo, 0, row0 / a.rgroup, zc0 + 2 * pair, &bar[0]);
      }
    };
    // thread 0's bounded wait for the pair; the CTA reads the outcome after its
    // next barrier and then acquires the pair with a wait that returns at once
    auto wait_start = [&]() {
      if (tid == 0) *flag = mbar_wait(&bar[0], phase, a.wait_limit) ? 0 : 1;
    };
    auto wait_finish = [&]() -> bool {
      const unsigned par = phase;
      phase ^= 1u;
      if (*flag) return false;
      mbar_wait(&bar[0], par, a.wait_limit);
      return true;
    };
    // primitives of the staged cell at raw offset o
    auto cell_prim = [&](int o, R (&V)[NV]) {
      const R *r = rawcc;
      if constexpr (MHD) {
        float u[8];
#pragma unroll
        for (int v = 0; v < 8; v++) u[v] = r[v * RV + o];
        slab_prim_mhd(a.gm1, u, rawlo[o], V);
      } else if constexpr (LO) {
        slab_prim(a.gm1, r[o], r[RV + o], r[2 * RV + o], r[3 * RV + o], r[4 * RV + o], rawlo[o], V);
      } else {
        slab_prim(a.eos, r[o], r[RV + o], r[2 * RV + o], r[3 * RV + o], r[4 * RV + o], V);
      }
    };
    // own column of a pair -> primitives (a pair over the two planes)
    auto convert_own = [&](P (&W)[NV], bool keep) {
      const int o = (wr + HH) * np0 + lane + gx;
      R V0[NV], V1[NV];
      cell_prim(o, V0);
      cell_prim(RPL + o, V1);
#pragma unroll
      for (int v = 0; v < NV; v++) W[v] = mk2(V0[v], V1[v]);
      if (keep) {
#pragma unroll
        for (int v = 0; v < NV; v++) prim[(v * PR + wr + HH) * PC + lane + HH] = W[v];
      }
    };
    // the x and y halo cells of a centre pair
    auto convert_halo = [&]() {
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
        R V0[NV], V1[NV];
        cell_prim(o, V0);
        cell_prim(RPL + o, V1);
#pragma unroll
        for (int v = 0; v < NV; v++) prim[(v * PR + rr) * PC + cc] = mk2(V0[v], V1[v]);
      }
    };
    // constrained transport: face-array offsets of this block (interior
    // coordinates), and the transverse field fluxes of a face pair written
    // for the edge EMFs (each face by the tile that owns it)
    int kz = 0;  // the current pair's first plane
    const long long NF = (long long)m.nb * m.Pf, fbo = (long long)b * m.Pf;
    const long long fsk = (long long)m.nf[0] * m.nf[1];
    auto foff = [&](int k, int jj, int ii) {
      return fbo + ((long long)(k + m.g[2]) * m.nf[1] + (jj + m.g[1])) * m.nf[0] + (ii + m.g[0]);
    };
    auto put_bt = [&](int dir, long long fo, const float (&Bt)[2][2], bool own0, bool own1) {
      if constexpr (MHD) {
        const int t0 = dir == 0 ? 1 : 0, t1 = dir == 2 ? 1 : 2;
        R *F0 = a.flux + ((long long)dir * 8 + CMAGC0 + t0) * NF;
        R *F1 = a.flux + ((long long)dir * 8 + CMAGC0 + t1) * NF;
        if (own0) {
          F0[fo] = Bt[0][0];
          F1[fo] = Bt[0][1];
        }
        if (own1) {
          F0[fo + fsk] = Bt[1][0];
          F1[fo + fsk] = Bt[1][1];
        }
      }
    };
    auto recon_x = [&](int v, int r, int xx) {
      const P *c = prim + (v * PR + r + HH) * PC + xx;
      P s[5];
#pragma unroll
      for (int q = 0; q < 5; q++) s[q] = c[q];
      P vm, vp;
      ReconPair<RECON>(a.limiter, s, vm, vp);
      rm[v * REC_N + r * RXC + xx] = vm;
      rp[v * REC_N + r * RXC + xx] = vp;
    };
    auto riemann_x = [&](int r, int f) {
      P vL[NV], vR[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        vL[v] = rp[v * REC_N + r * RXC + f];
        vR[v] = rm[v * REC_N + r * RXC + f + 1];
      }
      P F[NCV];
      if constexpr (MHD) {
        // x face f of tile row r on the pair's two planes; every one is this tile's
        const long long fo = foff(kz, oy + r, f);
        float Bt[2][2];
        SlabRiemannMHD2<RIEMANN, 0>(vL, vR, a.gam, mk2(a.fc0[fo], a.fc0[fo + fsk]), F, Bt);
        put_bt(0, fo, Bt, true, true);
      } else {
        SlabRiemann2<RIEMANN, 0>(vL, vR, a.gam, F);
      }
#pragma unroll
      for (int v = 0; v < NCV; v++) flx[v * FLX_N + r * (NX + 1) + f] = F[v];
    };
    auto recon_y = [&](int v, int yy, int x) {
      const P *c = prim + (v * PR + yy) * PC + x + HH;
      P s[5];
#pragma unroll
      for (int q = 0; q < 5; q++) s[q] = c[q * PC];
      P vm, vp;
      ReconPair<RECON>(a.limiter, s, vm, vp);
      rm[v * REC_N + yy * NX + x] = vm;
      rp[v * REC_N + yy * NX + x] = vp;
    };
    auto riemann_y = [&](int f, int x) {
      P vL[NV], vR[NV];
#pragma unroll
      for (int v = 0; v < NV; v++) {
        vL[v] = rp[v * REC_N + f * NX + x];
        vR[v] = rm[v * REC_N + (f + 1) * NX + x];
      }
      P F[NCV];
      if constexpr (MHD) {
        // y face oy + f: the tile's own unless it is the next tile's first row
        const long long fo = foff(kz, oy + f, x);
        float Bt[2][2];
        SlabRiemannMHD2<RIEMANN, 1>(vL, vR, a.gam, mk2(a.fc0[NF + fo], a.fc0[NF + fo + fsk]), F, Bt);
        const bool own = f < TY || oy + TY == m.nx[1];
        put_bt(1, fo, Bt, own, own);
      } else {
        SlabRiemann2<RIEMANN, 1>(vL, vR, a.gam, F);
      }
#pragma unroll
      for (int v = 0; v < NCV; v++) flx[v * FLX_N + f * NX + x] = F[v];
    };

    // z window: planes (2j-2, 2j-1), (2j, 2j+1).  Carried between steps:
    // vPc = z face value vP of cell 2j-1; Fc = z flux at face 2j-3/2 and
    // duc = x+y divergence of cell 2j-1 (both for the pending update of cell
    // 2j-1); du = x+y divergence of the step's planes (y part added in the
    // next step's first phase); zF = the step's z fluxes.
    P W0[NV], W1[NV];
    R vPc[NV], Fc[NCV], duc[NCV];
    P du[NCV], zF[NCV];
#pragma unroll
    for (int v = 0; v < NV; v++) vPc[v] = R(0);
#pragma unroll
    for (int v = 0; v < NCV; v++) {
      Fc[v] = duc[v] = R(0);
      du[v] = zF[v] = splat(R(0));
    }

    // inputs of the pending update (cells 2j-3, 2j-2 at step j), loaded at the
    // end of the previous step so the loads complete during its last barrier
    bool ok[2] = {false, false};
    long long n[2] = {0, 0};
    R zb[2][NCV], z0[2][NCV];
    float zblo[2], z0lo[2];
    auto load_update = [&](int zlo) {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int z = zlo + h;
        ok[h] = z >= 0 && z < nz;
        n[h] = col + (long long)(z + m.g[2]) * plane_st;
        if (ok[h]) {
#pragma unroll
          for (int v = 0; v < NCV; v++) {
            zb[h][v] = a.ub[v * NP + n[h]];
            z0[h][v] = a.u0[v * NP + n[h]];
          }
          if constexpr (LO) {
            zblo[h] = a.ublo[n[h]];
            z0lo[h] = a.u0lo[n[h]];
          }
        }
      }
    };

    issue(-2);
    wait_start();
    __syncthreads();
    if (!wait_finish()) {
      failed = true;
      break;
    }
    convert_own(W0, false);
    __syncthreads();
    issue(-1);
    wait_start();
    __syncthreads();
    if (!wait_finish()) {
      failed = true;
      break;
    }
    convert_own(W1, false);
    __syncthreads();

    for (int j = -1; j <= nz2 + 1; j++) {
      const bool centre = j >= 0 && j < nz2;
      kz = 2 * j;
      // ---- phase A: the pending update of cells (2j-3, 2j-2), the next
      // pair's loads, x reconstruction of this step's planes ----
      if (j - 1 >= 0 && j - 1 < nz2) {
        // y divergence of step j-1's planes
#pragma unroll
        for (int v = 0; v < NCV; v++) {
          const P lo = flx[v * FLX_N + wr * NX + lane], hi = flx[v * FLX_N + (wr + 1) * NX + lane];
          du[v] = psub2(du[v], psub2(pmul(splat(A1), hi), pmul(splat(A1), lo)));
        }
      }
      if (j >= 1) {
        R dz[2][NCV];
#pragma unroll
        for (int v = 0; v < NCV; v++) {
          // z contributions -A (F+ - F-) after x and y, as the reference sums them
          dz[0][v] = duc[v] - (A2 * zF[v].x - A2 * Fc[v]);
          dz[1][v] = du[v].x - (A2 * zF[v].y - A2 * zF[v].x);
        }
        const int zlo = 2 * j - 3;
#pragma unroll
        for (int h = 0; h < 2; h++) {
          if (!ok[h]) continue;
          GhostVal<R> gv;
          gv.lo = 0.f;
#pragma unroll
          for (int v = 0; v < NCV; v++) {
            const R dudt = dz[h][v] / vol;
            if (LO && v == CENER) {
              // FP32: the energy in FP64 from its hi/lo words
              const double eb = double(zb[h][v]) + double(zblo[h]), e0 = double(z0[h][v]) + double(z0lo[h]);
              const double e1 = (a.beta * eb + (1.0 - a.beta) * e0) + a.beta * dt * double(dudt);
              gv.v[v] = R(e1);
              gv.lo = float(e1 - double(gv.v[v]));
            } else {
              gv.v[v] = (bt * zb[h][v] + (R(1) - bt) * z0[h][v]) + bt * R(dt) * dudt;
            }
            a.u1[v * NP + n[h]] = gv.v[v];
          }
          if constexpr (LO) a.u1lo[n[h]] = gv.lo;
          // face ghosts: only where the cell lies within g of a block face
          const int z = zlo + h;
          const bool pz = z < m.g[2] || z >= nz - m.g[2];
          if (px | py | pz) {
            const int pc[3] = {lane + gx, oy + wr + m.g[1], z + m.g[2]};
            if (px) ghost_push_axis(a, 0, b, lb, pc, gv);
            if (py) ghost_push_axis(a, 1, b, lb, pc, gv);
            if (pz) ghost_push_axis(a, 2, b, lb, pc, gv);
          }
          // (constrained transport: the cell pass after the face update takes the estimate)
          if (!MHD && a.last) {
            if constexpr (MHD) {
            } else if constexpr (LO) {
              float V[NV];
              slab_prim(a.gm1, gv.v[0], gv.v[1], gv.v[2], gv.v[3], gv.v[4], gv.lo, V);
#pragma unroll
              for (int d = 0; d < 3; d++) {
                const float cf = sqrtf(a.gam * V[SPRES] / V[SD]);
                double xv = double(float(m.dx[d]) / (fabsf(V[SV0 + d]) + cf));
                if (xv != xv) xv = 0.0;
                dtl = xv < dtl ? xv : dtl;
              }
            } else {
              // hydro_time_step.cpp:19-64 as the other FP64 stages evaluate it
              double V[7];
              Cons2PrimEos<false, double>(a.eos, gv.v[0], gv.v[1], gv.v[2], gv.v[3], gv.v[4], nullptr, V);
#pragma unroll
              for (int d = 0; d < 3; d++) {
                const double cf = FastSpeed<false>(d, V);
                double xv = m.dx[d] / (fabs(V[RVEL0 + d]) + cf);
                if (xv != xv) xv = 0.0;
                dtl = xv < dtl ? xv : dtl;
              }
            }
          }
        }
      }
      if (j > nz2) break;
      // the pending update of cell 2j-1 in the next step takes these
#pragma unroll
      for (int v = 0; v < NCV; v++) {
        Fc[v] = zF[v].y;
        duc[v] = du[v].y;
        du[v] = splat(R(0));
      }
      issue(j + 1);
      if (centre) {
#pragma unroll(RU)
        for (int v = 0; v < NV; v++) recon_x(v, wr, lane);
        if (tid < NV * TY * 2) recon_x(tid / (2 * TY), (tid % (2 * TY)) >> 1, NX + (tid & 1));
      }
      __syncthreads();
      // ---- phase B: x Riemann fluxes ----
      if (centre) {
        riemann_x(wr, lane);
        if (tid < TY) riemann_x(tid, NX);
      }
      __syncthreads();
      // ---- phase C: x divergence, y reconstruction, wait for the next pair ----
      if (centre) {
#pragma unroll
        for (int v = 0; v < NCV; v++) {
          const P lo = flx[v * FLX_N + wr * (NX + 1) + lane], hi = flx[v * FLX_N + wr * (NX + 1) + lane + 1];
          du[v] = psub2(du[v], psub2(pmul(splat(A0), hi), pmul(splat(A0), lo)));
        }
#pragma unroll(RU)
        for (int v = 0; v < NV; v++) recon_y(v, wr, lane);
        for (int it = tid; it < NV * 2 * NX; it += NT) recon_y(it >> 6, TY + ((it >> 5) & 1), lane);
      }
      wait_start();
      __syncthreads();
      // ---- phase D: y Riemann fluxes, the next pair's primitives, the z sweep ----
      if (!wait_finish()) {
        failed = true;
        break;
      }
      if (centre) {
        riemann_y(wr, lane);
        // the extra face row on the last warp: the first warps also convert
        // the next pair's halo cells in this phase
#if SLAB_Y_EXTRAS_LAST_WARP
        if (tid >= NT - NX) riemann_y(TY, tid - (NT - NX));
#else
        if (tid < NX) riemann_y(TY, tid);
#endif
      }
      const bool next_centre = j + 1 >= 0 && j + 1 < nz2;
      P W2[NV];
      convert_own(W2, next_centre);
      if (next_centre) convert_halo();
      {
        // cells (2j, 2j+1) of the column, faces 2j - 1/2 and 2j + 1/2
        P vm[NV], vp[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) {
          const P s[5] = {W0[v], mk2(W0[v].y, W1[v].x), W1[v], mk2(W1[v].y, W2[v].x), W2[v]};
          ReconPair<RECON>(a.limiter, s, vm[v], vp[v]);
        }
        P vL[NV];
#pragma unroll
        for (int v = 0; v < NV; v++) vL[v] = mk2(vPc[v], vp[v].x);
        if constexpr (MHD) {
          // z faces 2j and 2j + 1 of the column; those in 0 .. nz are its own
          const long long fo = foff(2 * j, oy + wr, lane);
          float Bt[2][2];
          SlabRiemannMHD2<RIEMANN, 2>(vL, vm, a.gam, mk2(a.fc0[2 * NF + fo], a.fc0[2 * NF + fo + fsk]), zF, Bt);
          put_bt(2, fo, Bt, 2 * j >= 0 && 2 * j <= nz, 2 * j + 1 >= 0 && 2 * j + 1 <= nz);
        } else {
          SlabRiemann2<RIEMANN, 2>(vL, vm, a.gam, zF);
        }
#pragma unroll
        for (int v = 0; v < NV; v++) {
          vPc[v] = vp[v].y;
          W0[v] = W1[v];
          W1[v] = W2[v];
        }
      }
      load_update(2 * j - 1);
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

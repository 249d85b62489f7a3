// kmy_device.cuh -- per-cell / per-face arithmetic of the hydro update.
//
// Device restatements of the reference's inline functions, templated on the
// arithmetic type R (double for the FP64 path, float for the FP32 bulk path).
// Expressions keep the reference's operation order; nvcc may contract a*b+c
// into FMA, which moves results by at most an ulp per operation.
#pragma once

#include <cfloat>
#include <cstdint>

namespace kmy {

enum Recon : int { FOG = 0, PLM = 1, PPM = 2, WENOZ = 3 };
enum Limiter : int { MINMOD = 0, VAN_LEER = 1, MC = 2 };
enum RiemannSolver : int { HLL = 0, HLLC = 1 };
enum BoundaryKind : int { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2 };

// slots of a conserved state
enum : int { CDENS = 0, CMOM0 = 1, CMOM1 = 2, CMOM2 = 3, CENER = 4, CMAGC0 = 5 };
// slots of a reconstructed (primitive) state, hydro_types.hpp:61-77 order
enum : int { RDENS = 0, RVEL0 = 1, RVEL1 = 2, RVEL2 = 3, RPRES = 4, RBMOD = 5, REINT = 6, RMAGC0 = 7 };
// shared primitive arrays in device storage (density lives with the conserved)
enum : int { PVEL0 = 0, PVEL1 = 1, PVEL2 = 2, PPRES = 3, PBMOD = 4, PEINT = 5, PTEMP = 6, NPRIM = 7 };

template <typename R> struct Lim;
template <> struct Lim<double> {
  static __host__ __device__ constexpr double tiny() { return DBL_MIN; }
};
template <> struct Lim<float> {
  static __host__ __device__ constexpr float tiny() { return FLT_MIN; }
};

template <typename R> __device__ __forceinline__ R kmin(R a, R b) { return (b < a) ? b : a; }
template <typename R> __device__ __forceinline__ R kmax(R a, R b) { return (a < b) ? b : a; }
template <typename R> __device__ __forceinline__ R sq(R x) { return x * x; }

// FP64 reciprocal by Newton-Raphson: the hardware approximation
// (rcp.approx.ftz.f64, PTX ISA) refined by two iterations r <- r + r (1 - x r),
// each of which squares the relative error, so the result is within an ulp or
// two of 1/x for finite, nonzero, normal x (tests/test_gpu_kat.py holds it to
// 2 ulps of IEEE 1/x).  It takes two fewer dependent FP64 operations than
// IEEE division and no slow-path branch.  Zero and infinite x give NaN (IEEE
// division gives inf and 0): only states that are already not physical reach
// them, and the dt controller reports those as non-finite.
__device__ __forceinline__ double rcp_nr(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  r = fma(r, fma(-x, r, 1.0), r);
  return fma(r, fma(-x, r, 1.0), r);
}
// FP64 square root by Newton-Raphson on the reciprocal square root: the
// hardware approximation (rsqrt.approx.ftz.f64) refined by two iterations
// y <- y (3/2 - a y^2 / 2), then sqrt(a) = a y, within 3 ulps of IEEE sqrt
// for normal a > 0 (tests/test_gpu_kat.py); sqrt(0) = 0 and negative a gives
// NaN, as IEEE sqrt does.
__device__ __forceinline__ double sqrt_nr(double a) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  const double h = 0.5 * a;
  y = y * fma(-h, y * y, 1.5);
  y = y * fma(-h, y * y, 1.5);
  return a == 0.0 ? a : a * y;
}

// Division and square root of the per-cell arithmetic below.  A unit that
// defines KMY_F64_NR as 1 before including this header (the FP64 brick and
// batched stages) takes the Newton-Raphson forms above in FP64; every other
// unit (the per-task kernels among them), and FP32 everywhere, takes a / b and
// sqrt(a) as the unit's compiler flags round them.
#ifndef KMY_F64_NR
#define KMY_F64_NR 0
#endif
template <typename R> __device__ __forceinline__ R kdiv(R a, R b) {
  if constexpr (KMY_F64_NR && sizeof(R) == sizeof(double)) return a * rcp_nr(b);
  else return a / b;
}
template <typename R> __device__ __forceinline__ R ksqrt(R a) {
  if constexpr (KMY_F64_NR && sizeof(R) == sizeof(double)) return sqrt_nr(a);
  else return sqrt(a);
}

// reconstruction.hpp:24-39
template <typename R>
__device__ __forceinline__ R LimitedSlope(int limiter, R a, R b) {
  if (limiter == MC) {
    return (copysign(R(1), a) + copysign(R(1), b)) *
           kmin(fabs(a), kmin(R(.25) * fabs(a + b), fabs(b)));
  } else if (limiter == VAN_LEER) {
    if (a * b > R(0)) return kdiv(R(2) * a * b, a + b);
    return R(0);
  }
  return R(0.5) * (copysign(R(1), a) + copysign(R(1), b)) * kmin(fabs(a), fabs(b));
}

// Stencil half-width each reconstruction reads (cells c-W .. c+W).
template <int RECON> struct ReconWidth { static constexpr int value = 0; };
template <> struct ReconWidth<PLM> { static constexpr int value = 1; };
template <> struct ReconWidth<PPM> { static constexpr int value = 2; };
template <> struct ReconWidth<WENOZ> { static constexpr int value = 2; };

__host__ __device__ inline int ReconWidthRuntime(int recon) {
  return recon == FOG ? 0 : recon == PLM ? 1 : 2;
}

// WENO-Z weight factor 1 + (tau/(eps + beta))^2 (reconstruction.hpp:118-135).
// In FP32 the ratio is capped at 1e15 so its square stays finite: with
// eps = 1e-36 a vanishing smoothness indicator gives ratios far beyond the
// float range, and at 1e15 that stencil already holds the whole weight.
template <typename R>
__device__ __forceinline__ R weno_q(R tau, R beta) {
  R r = kdiv(tau, R(1.e-36) + beta);
  if constexpr (sizeof(R) == 4) r = fminf(r, 1.0e15f);
  return R(1) + sq(r);
}

// reconstruction.hpp:11-142: both face values of the cell at s[0] (s indexed
// -W..W through the pointer arithmetic of the caller: s[o] = value at c+o).
template <int RECON, typename R>
__device__ __forceinline__ void Reconstruct(int limiter, const R (&s)[5], R &vM, R &vP) {
  // s[0..4] hold offsets -2..2
  const R s0 = s[2];
  if constexpr (RECON == FOG) {
    vM = s0;
    vP = s0;
  } else if constexpr (RECON == PLM) {
    const R dvL = s0 - s[1];
    const R dvR = s[3] - s0;
    const R del = LimitedSlope(limiter, dvL, dvR);
    vM = s0 - R(0.5) * del;
    vP = s0 + R(0.5) * del;
  } else if constexpr (RECON == PPM) {
    const R dv_p = LimitedSlope(limiter, s[4] - s[3], s[3] - s0);
    const R dv_0 = LimitedSlope(limiter, s[3] - s0, s0 - s[1]);
    const R dv_m = LimitedSlope(limiter, s0 - s[1], s[1] - s[0]);
    const R sixth = R(1.) / R(6.);
    vM = R(0.5) * (s[1] + s0) - sixth * (dv_0 - dv_m);
    vP = R(0.5) * (s0 + s[3]) - sixth * (dv_p - dv_0);
    if ((vP - s0) * (s0 - vM) <= R(0)) {
      vM = s0;
      vP = s0;
    }
    if (-(vP - vM) * (vP - vM) > R(6) * (vP - vM) * (s0 - R(0.5) * (vP + vM))) {
      vP = R(3) * s0 - R(2) * vM;
    }
    if ((vP - vM) * (vP - vM) < R(6) * (vP - vM) * (s0 - R(0.5) * (vP + vM))) {
      vM = R(3) * s0 - R(2) * vP;
    }
  } else {
    const R sixth = R(1.) / R(6.);
    // eno predictions at +1/2 (pm=+1) and -1/2 (pm=-1)
    const R ep0 = sixth * (-s[4] + R(5) * s[3] + R(2) * s0);
    const R ep1 = sixth * (R(2) * s[3] + R(5) * s0 - s[1]);
    const R ep2 = sixth * (R(11) * s0 - R(7) * s[1] + R(2) * s[0]);
    const R em0 = sixth * (-s[0] + R(5) * s[1] + R(2) * s0);
    const R em1 = sixth * (R(2) * s[1] + R(5) * s0 - s[3]);
    const R em2 = sixth * (R(11) * s0 - R(7) * s[3] + R(2) * s[4]);
    const R c1312 = R(13.) / R(12.);
    const R b0 = c1312 * sq(s[0] - R(2) * s[1] + s0) + R(0.25) * sq(s[0] - R(4) * s[1] + R(3) * s0);
    const R b1 = c1312 * sq(s[1] - R(2) * s0 + s[3]) + R(0.25) * sq(s[1] - s[3]);
    const R b2 = c1312 * sq(s0 - R(2) * s[3] + s[4]) + R(0.25) * sq(s[4] - R(4) * s[3] + R(3) * s0);
    const R eps = R(1.e-36);
    const R tau = fabs(b2 - b0);
    (void)eps;
    const R q0 = weno_q(tau, b0);
    const R q1 = weno_q(tau, b1);
    const R q2 = weno_q(tau, b2);
    {  // pm = -1: w0 uses beta0, w2 uses beta2
      const R w0 = R(3) * q0, w1 = R(6) * q1, w2 = R(1) * q2;
      const R norm = w0 + w1 + w2;
      vM = kdiv(w0 * em0 + w1 * em1 + w2 * em2, norm);
    }
    {  // pm = +1: w0 uses beta2, w2 uses beta0
      const R w0 = R(3) * q2, w1 = R(6) * q1, w2 = R(1) * q0;
      const R norm = w0 + w1 + w2;
      vP = kdiv(w0 * ep0 + w1 * ep1 + w2 * ep2, norm);
    }
  }
}

// WENO-Z at both faces with two divisions instead of five (FP64 fused
// stage).  The reference's weights w_k = d_k (1 + tau^2 / A_k), with
// A_k = (eps + beta_k)^2, are scaled by A_0 A_1 A_2, which the normalisation
// cancels: W_k = d_k (A_k + tau^2) prod_{j != k} A_j.  Same value as
// Reconstruct up to rounding; with eps = 1e-36 the scaled weights stay
// within [1e-216, 1e+216] for smoothness indicators up to 1e+36.
// The two divisions as the unit's kdiv by default; a stage may pass its own
// form: DivIeee (a / b) or DivNR (a times the Newton-Raphson reciprocal).
struct DivIeee {
  template <typename R>
  static __device__ __forceinline__ R div(R a, R b) { return a / b; }
};
struct DivNR {
  static __device__ __forceinline__ double div(double a, double b) { return a * rcp_nr(b); }
};
struct DivK {
  template <typename R>
  static __device__ __forceinline__ R div(R a, R b) { return kdiv(a, b); }
};

template <typename R, typename Div = DivK>
__device__ __forceinline__ void WenoZBothTwoDiv(const R (&s)[5], R &vM, R &vP) {
  const R s0 = s[2];
  const R sixth = R(1.) / R(6.);
  const R ep0 = sixth * (-s[4] + R(5) * s[3] + R(2) * s0);
  const R ep1 = sixth * (R(2) * s[3] + R(5) * s0 - s[1]);
  const R ep2 = sixth * (R(11) * s0 - R(7) * s[1] + R(2) * s[0]);
  const R em0 = sixth * (-s[0] + R(5) * s[1] + R(2) * s0);
  const R em1 = sixth * (R(2) * s[1] + R(5) * s0 - s[3]);
  const R em2 = sixth * (R(11) * s0 - R(7) * s[3] + R(2) * s[4]);
  const R c1312 = R(13.) / R(12.);
  const R b0 = c1312 * sq(s[0] - R(2) * s[1] + s0) + R(0.25) * sq(s[0] - R(4) * s[1] + R(3) * s0);
  const R b1 = c1312 * sq(s[1] - R(2) * s0 + s[3]) + R(0.25) * sq(s[1] - s[3]);
  const R b2 = c1312 * sq(s0 - R(2) * s[3] + s[4]) + R(0.25) * sq(s[4] - R(4) * s[3] + R(3) * s0);
  const R t2 = sq(b2 - b0);
  const R A0 = sq(R(1.e-36) + b0), A1 = sq(R(1.e-36) + b1), A2 = sq(R(1.e-36) + b2);
  const R N0 = A0 + t2, N1 = A1 + t2, N2 = A2 + t2;
  const R P01 = A0 * A1, P02 = A0 * A2, P12 = A1 * A2;
  {  // minus face: d = (3, 6, 1) on (beta0, beta1, beta2)
    const R w0 = R(3) * N0 * P12, w1 = R(6) * N1 * P02, w2 = N2 * P01;
    vM = Div::div(w0 * em0 + w1 * em1 + w2 * em2, w0 + w1 + w2);
  }
  {  // plus face: d = (3, 6, 1) on (beta2, beta1, beta0)
    const R w0 = R(3) * N2 * P01, w1 = R(6) * N1 * P02, w2 = N0 * P12;
    vP = Div::div(w0 * ep0 + w1 * ep1 + w2 * ep2, w0 + w1 + w2);
  }
}

// ---------------------------------------------------------------------------
// Packed FP32.  sm_100 issues one add, multiply or fma instruction for both
// lanes of a float2, so the FP32 fused stage reconstructs two cells per
// thread.  Reciprocals stay per lane (rcp.approx on the XU pipe).
__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float2 prcp(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }

// WENO-Z weight factor on two lanes: 1 + min((tau/(eps+beta))^2, 1e30).
// Capping the square at 1e30 is the FP32 cap of the ratio at 1e15 (weno_q),
// and tau's sign drops out of the square, so tau may be b2 - b0 unsigned.
__device__ __forceinline__ float2 weno_q2(float2 tau, float2 beta) {
  const float2 r = pmul(tau, prcp(padd(p2(1.e-36f), beta)));
  float2 r2 = pmul(r, r);
  r2.x = fminf(r2.x, 1.0e30f);
  r2.y = fminf(r2.y, 1.0e30f);
  return padd(p2(1.f), r2);
}

// WENO-Z at both faces of two cells (reconstruction.hpp:104-142): the
// reference's candidate stencils, smoothness indicators and weights, with
// the 1/6 of the candidates folded into their coefficients and the
// normalisation done by one reciprocal per face value.
__device__ __forceinline__ void WenoZBoth2(const float2 (&s)[5], float2 &vM, float2 &vP) {
  const float2 a = s[0], b = s[1], c = s[2], d = s[3], e = s[4];
  const float2 c2 = pmul(p2(2.f / 6.f), c), c5 = pmul(p2(5.f / 6.f), c), c11 = pmul(p2(11.f / 6.f), c);
  const float2 ep0 = pfma(p2(-1.f / 6.f), e, pfma(p2(5.f / 6.f), d, c2));
  const float2 em0 = pfma(p2(-1.f / 6.f), a, pfma(p2(5.f / 6.f), b, c2));
  const float2 ep1 = pfma(p2(2.f / 6.f), d, pfma(p2(-1.f / 6.f), b, c5));
  const float2 em1 = pfma(p2(2.f / 6.f), b, pfma(p2(-1.f / 6.f), d, c5));
  const float2 ep2 = pfma(p2(-7.f / 6.f), b, pfma(p2(2.f / 6.f), a, c11));
  const float2 em2 = pfma(p2(-7.f / 6.f), d, pfma(p2(2.f / 6.f), e, c11));
  const float2 k1 = p2(13.f / 12.f), k2 = p2(0.25f);
  const float2 c3 = pmul(p2(3.f), c);
  const float2 u0 = pfma(p2(-2.f), b, padd(a, c)), v0 = pfma(p2(-4.f), b, padd(a, c3));
  const float2 u1 = pfma(p2(-2.f), c, padd(b, d)), v1 = pfma(p2(-1.f), d, b);
  const float2 u2 = pfma(p2(-2.f), d, padd(c, e)), v2 = pfma(p2(-4.f), d, padd(e, c3));
  const float2 b0 = pfma(pmul(k1, u0), u0, pmul(pmul(k2, v0), v0));
  const float2 b1 = pfma(pmul(k1, u1), u1, pmul(pmul(k2, v1), v1));
  const float2 b2 = pfma(pmul(k1, u2), u2, pmul(pmul(k2, v2), v2));
  const float2 tau = pfma(p2(-1.f), b0, b2);
  const float2 q0 = weno_q2(tau, b0), q1 = weno_q2(tau, b1), q2 = weno_q2(tau, b2);
  const float2 t0 = pmul(p2(3.f), q0), t1 = pmul(p2(6.f), q1), t2 = pmul(p2(3.f), q2);
  // minus face: w = (3 q0, 6 q1, q2); plus face: w = (3 q2, 6 q1, q0)
  vM = pmul(pfma(t0, em0, pfma(t1, em1, pmul(q2, em2))), prcp(padd(t0, padd(t1, q2))));
  vP = pmul(pfma(t2, ep0, pfma(t1, ep1, pmul(q0, ep2))), prcp(padd(t2, padd(t1, q0))));
}

// Both face values of two cells: packed WENO-Z, else the scalar
// reconstruction once per lane (bit-identical to Reconstruct).
template <int RECON>
__device__ __forceinline__ void ReconstructBoth2(int limiter, const float2 (&s)[5], float2 &vM, float2 &vP) {
  if constexpr (RECON == WENOZ) {
    WenoZBoth2(s, vM, vP);
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

// Value at the plus face only (for the cell left of a face).
template <int RECON, typename R>
__device__ __forceinline__ R ReconstructPlus(int limiter, const R (&s)[5]) {
  if constexpr (RECON == WENOZ) {
    const R s0 = s[2];
    const R sixth = R(1.) / R(6.);
    const R ep0 = sixth * (-s[4] + R(5) * s[3] + R(2) * s0);
    const R ep1 = sixth * (R(2) * s[3] + R(5) * s0 - s[1]);
    const R ep2 = sixth * (R(11) * s0 - R(7) * s[1] + R(2) * s[0]);
    const R c1312 = R(13.) / R(12.);
    const R b0 = c1312 * sq(s[0] - R(2) * s[1] + s0) + R(0.25) * sq(s[0] - R(4) * s[1] + R(3) * s0);
    const R b1 = c1312 * sq(s[1] - R(2) * s0 + s[3]) + R(0.25) * sq(s[1] - s[3]);
    const R b2 = c1312 * sq(s0 - R(2) * s[3] + s[4]) + R(0.25) * sq(s[4] - R(4) * s[3] + R(3) * s0);
    const R eps = R(1.e-36);
    const R tau = fabs(b2 - b0);
    (void)eps;
    const R w0 = R(3) * weno_q(tau, b2);
    const R w1 = R(6) * weno_q(tau, b1);
    const R w2 = R(1) * weno_q(tau, b0);
    const R norm = w0 + w1 + w2;
    return (w0 * ep0 + w1 * ep1 + w2 * ep2) / norm;
  } else {
    R vM, vP;
    Reconstruct<RECON, R>(limiter, s, vM, vP);
    return vP;
  }
}

// Value at the minus face only (for the cell right of a face).
template <int RECON, typename R>
__device__ __forceinline__ R ReconstructMinus(int limiter, const R (&s)[5]) {
  if constexpr (RECON == WENOZ) {
    const R s0 = s[2];
    const R sixth = R(1.) / R(6.);
    const R em0 = sixth * (-s[0] + R(5) * s[1] + R(2) * s0);
    const R em1 = sixth * (R(2) * s[1] + R(5) * s0 - s[3]);
    const R em2 = sixth * (R(11) * s0 - R(7) * s[3] + R(2) * s[4]);
    const R c1312 = R(13.) / R(12.);
    const R b0 = c1312 * sq(s[0] - R(2) * s[1] + s0) + R(0.25) * sq(s[0] - R(4) * s[1] + R(3) * s0);
    const R b1 = c1312 * sq(s[1] - R(2) * s0 + s[3]) + R(0.25) * sq(s[1] - s[3]);
    const R b2 = c1312 * sq(s0 - R(2) * s[3] + s[4]) + R(0.25) * sq(s[4] - R(4) * s[3] + R(3) * s0);
    const R eps = R(1.e-36);
    const R tau = fabs(b2 - b0);
    (void)eps;
    const R w0 = R(3) * weno_q(tau, b0);
    const R w1 = R(6) * weno_q(tau, b1);
    const R w2 = R(1) * weno_q(tau, b2);
    const R norm = w0 + w1 + w2;
    return (w0 * em0 + w1 * em1 + w2 * em2) / norm;
  } else {
    R vM, vP;
    Reconstruct<RECON, R>(limiter, s, vM, vP);
    return vM;
  }
}

// ---------------------------------------------------------------------------
// primconsflux.hpp:21-138 on register states.  V: reconstructed layout
// (RDENS..REINT [+RMAGC0..2]); U/F: conserved layout (CDENS..CENER [+CMAGC0..2]).
template <bool MHD, typename R>
__device__ __forceinline__ R TotalPres(const R *V) {
  R pres = V[RPRES];
  if constexpr (MHD) {
    pres += R(0.5) * (V[RMAGC0] * V[RMAGC0] + V[RMAGC0 + 1] * V[RMAGC0 + 1] +
                      V[RMAGC0 + 2] * V[RMAGC0 + 2]);
  }
  return pres;
}

template <bool MHD, typename R>
__device__ __forceinline__ R FastSpeed(int dir1, const R *V) {
  const R idens = kdiv(R(1.), V[RDENS]);
  const R a2 = idens * V[RBMOD];
  R cfast2;
  if constexpr (!MHD) {
    cfast2 = a2;
  } else {
    const R bb2 = V[RMAGC0 + dir1] * V[RMAGC0 + dir1] * idens;
    R b2 = R(0);
    for (int dir = 0; dir < 3; dir++) b2 += V[RMAGC0 + dir] * V[RMAGC0 + dir];
    b2 *= idens;
    cfast2 = R(0.5) * ((a2 + b2) + ksqrt((a2 - b2) * (a2 - b2) + R(4) * a2 * (b2 - bb2)));
  }
  return ksqrt(cfast2);
}

template <bool MHD, typename R>
__device__ __forceinline__ void Prim2Cons(const R *V, R *U) {
  U[CDENS] = V[RDENS];
  R emag = R(0), ekin = R(0);
#pragma unroll
  for (int dir = 0; dir < 3; dir++) {
    U[CMOM0 + dir] = V[RDENS] * V[RVEL0 + dir];
    ekin += V[RVEL0 + dir] * V[RVEL0 + dir];
    if constexpr (MHD) {
      U[CMAGC0 + dir] = V[RMAGC0 + dir];
      emag += V[RMAGC0 + dir] * V[RMAGC0 + dir];
    }
  }
  const R eint = V[REINT] * V[RDENS];
  ekin *= R(0.5) * V[RDENS];
  emag *= R(0.5);
  U[CENER] = eint + ekin + emag;
}

template <bool MHD, int DIR1, typename R>
__device__ __forceinline__ void Prim2Flux(const R *V, R *F) {
  constexpr int DIR2 = (DIR1 + 1) % 3;
  constexpr int DIR3 = (DIR1 + 2) % 3;
  F[CDENS] = V[RDENS] * V[RVEL0 + DIR1];
  R ptot = V[RPRES];
  R B2 = R(0), uB = R(0), ekin = R(0);
#pragma unroll
  for (int dir = 0; dir < 3; dir++) {
    F[CMOM0 + dir] = F[CDENS] * V[RVEL0 + dir];
    ekin += V[RVEL0 + dir] * V[RVEL0 + dir];
    if constexpr (MHD) {
      B2 += V[RMAGC0 + dir] * V[RMAGC0 + dir];
      uB += V[RVEL0 + dir] * V[RMAGC0 + dir];
      F[CMOM0 + dir] -= V[RMAGC0 + DIR1] * V[RMAGC0 + dir];
    }
  }
  ekin *= R(0.5) * V[RDENS];
  const R emag = R(0.5) * B2;
  ptot += R(0.5) * B2;
  const R etot = V[REINT] * V[RDENS] + ekin + emag;
  F[CMOM0 + DIR1] += ptot;
  F[CENER] = (etot + ptot) * V[RVEL0 + DIR1];
  if constexpr (MHD) {
    F[CENER] -= uB * V[RMAGC0 + DIR1];
    F[CMAGC0 + DIR1] = R(0);
    F[CMAGC0 + DIR2] = V[RVEL0 + DIR1] * V[RMAGC0 + DIR2] - V[RVEL0 + DIR2] * V[RMAGC0 + DIR1];
    F[CMAGC0 + DIR3] = V[RVEL0 + DIR1] * V[RMAGC0 + DIR3] - V[RVEL0 + DIR3] * V[RMAGC0 + DIR1];
  }
}

// riemann_solver.hpp:20-57 (HLL) and :59-149 (HLLC) for the face normal DIR1.
template <int RIEMANN, bool MHD, int DIR1, typename R>
__device__ __forceinline__ void RiemannFlux(const R *vL, const R *vR, R *flux) {
  constexpr int DIR2 = (DIR1 + 1) % 3;
  constexpr int DIR3 = (DIR1 + 2) % 3;
  constexpr int NC = MHD ? 8 : 5;
  const R cfL = FastSpeed<MHD>(DIR1, vL);
  const R cfR = FastSpeed<MHD>(DIR1, vR);
  const R tiny = Lim<R>::tiny();
  const R sL = kmin(-tiny, kmin(vL[RVEL0 + DIR1] - cfL, vR[RVEL0 + DIR1] - cfR));
  const R sR = kmax(tiny, kmax(vL[RVEL0 + DIR1] + cfL, vR[RVEL0 + DIR1] + cfR));
  const R sRmsLi = kdiv(R(1.0), sR - sL);
  R UL[NC], UR[NC], FL[NC], FR[NC];
  Prim2Cons<MHD>(vL, UL);
  Prim2Cons<MHD>(vR, UR);
  Prim2Flux<MHD, DIR1>(vR, FR);
  Prim2Flux<MHD, DIR1>(vL, FL);
  if constexpr (RIEMANN == HLL) {
#pragma unroll
    for (int v = 0; v < NC; v++)
      flux[v] = sRmsLi * (sR * FL[v] - sL * FR[v] + sR * sL * (UR[v] - UL[v]));
  } else {
    const R total_presL = TotalPres<MHD>(vL);
    const R total_presR = TotalPres<MHD>(vR);
    R ustar = total_presR - total_presL + UL[CMOM0 + DIR1] * (sL - vL[RVEL0 + DIR1]) -
              UR[CMOM0 + DIR1] * (sR - vR[RVEL0 + DIR1]);
    ustar = kdiv(ustar, vL[RDENS] * (sL - vL[RVEL0 + DIR1]) - vR[RDENS] * (sR - vR[RVEL0 + DIR1]));
    const R pstar =
        R(0.5) * (total_presL + total_presR +
                  vL[RDENS] * (sL - vL[RVEL0 + DIR1]) * (ustar - vL[RVEL0 + DIR1]) +
                  vR[RDENS] * (sR - vR[RVEL0 + DIR1]) * (ustar - vR[RVEL0 + DIR1]));
    R UsL[NC], UsR[NC];
    auto hllc_state = [&](R S, const R *U, R Pu, R *Us) {
      const R susi = kdiv(R(1.), S - ustar + tiny);
      Us[CDENS] = susi * (S * U[CDENS] - U[CMOM0 + DIR1]);
      Us[CMOM0 + DIR1] = Us[CDENS] * ustar;
      // U * Us_dens / U_dens with one shared ratio (one division instead of three)
      const R rho_ratio = kdiv(Us[CDENS], U[CDENS]);
      Us[CMOM0 + DIR2] = U[CMOM0 + DIR2] * rho_ratio;
      Us[CMOM0 + DIR3] = U[CMOM0 + DIR3] * rho_ratio;
      Us[CENER] = U[CENER] * rho_ratio + susi * (pstar * ustar - Pu);
      if constexpr (MHD) {
        const R sRsLi = kdiv(R(1.), sR - sL);
        auto hll = [&](int v) { return sRsLi * (sR * UR[v] - sL * UL[v] + FL[v] - FR[v]); };
        Us[CMAGC0 + DIR1] = hll(CMAGC0 + DIR1);
        Us[CMAGC0 + DIR2] = hll(CMAGC0 + DIR2);
        Us[CMAGC0 + DIR3] = hll(CMAGC0 + DIR3);
        Us[CMOM0 + DIR2] -=
            (Us[CMAGC0 + DIR1] * Us[CMAGC0 + DIR2] - U[CMAGC0 + DIR1] * U[CMAGC0 + DIR2]) * susi;
        Us[CMOM0 + DIR3] -=
            (Us[CMAGC0 + DIR1] * Us[CMAGC0 + DIR3] - U[CMAGC0 + DIR1] * U[CMAGC0 + DIR3]) * susi;
        Us[CENER] -= susi * (kdiv(Us[CMAGC0 + DIR1] *
                                      (Us[CMAGC0 + DIR1] * hll(CMOM0 + DIR1) +
                                       Us[CMAGC0 + DIR2] * hll(CMOM0 + DIR2) +
                                       Us[CMAGC0 + DIR3] * hll(CMOM0 + DIR3)),
                                  hll(CDENS)) -
                             kdiv(U[CMAGC0 + DIR1] *
                                      (U[CMAGC0 + DIR1] * U[CMOM0 + DIR1] +
                                       U[CMAGC0 + DIR2] * U[CMOM0 + DIR2] +
                                       U[CMAGC0 + DIR3] * U[CMOM0 + DIR3]),
                                  U[CDENS]));
      }
    };
    hllc_state(sL, UL, total_presL * vL[RVEL0 + DIR1], UsL);
    hllc_state(sR, UR, total_presR * vR[RVEL0 + DIR1], UsR);
    const R biasL = -kmin(-tiny, copysign(R(1), ustar));
    const R biasR = kmax(tiny, copysign(R(1), ustar));
#pragma unroll
    for (int v = 0; v < NC; v++)
      flux[v] = biasR * (FL[v] + sL * (UsL[v] - UL[v])) + biasL * (FR[v] + sR * (UsR[v] - UR[v]));
  }
}

// ---------------------------------------------------------------------------
// The hydro Riemann fluxes above on two faces at once (packed FP32, the FP32
// fused stage).  Same formulas as RiemannFlux<RIEMANN, false, DIR1>: HLL
// (riemann_solver.hpp:20-57) and HLLC with both star states blended by the
// sign of u* (:59-149); divisions are per-lane approximate reciprocals.
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return pfma(p2(-1.f), b, a); }

template <int DIR1>
__device__ __forceinline__ void Prim2ConsFlux2(const float2 *V, float2 *U, float2 *F) {
  const float2 rho = V[RDENS], un = V[RVEL0 + DIR1];
  const float2 vv = pfma(V[RVEL0 + 2], V[RVEL0 + 2], pfma(V[RVEL0 + 1], V[RVEL0 + 1], pmul(V[RVEL0], V[RVEL0])));
  U[CDENS] = rho;
  F[CDENS] = pmul(rho, un);
#pragma unroll
  for (int d = 0; d < 3; d++) {
    U[CMOM0 + d] = pmul(rho, V[RVEL0 + d]);
    F[CMOM0 + d] = pmul(F[CDENS], V[RVEL0 + d]);
  }
  U[CENER] = padd(pmul(V[REINT], rho), pmul(pmul(p2(0.5f), rho), vv));
  F[CMOM0 + DIR1] = padd(F[CMOM0 + DIR1], V[RPRES]);
  F[CENER] = pmul(padd(U[CENER], V[RPRES]), un);
}

template <int RIEMANN, int DIR1>
__device__ __forceinline__ void RiemannFlux2(const float2 *vL, const float2 *vR, float2 *flux) {
  constexpr int DIR2 = (DIR1 + 1) % 3;
  constexpr int DIR3 = (DIR1 + 2) % 3;
  const float tiny = FLT_MIN;
  const float2 uL = vL[RVEL0 + DIR1], uR = vR[RVEL0 + DIR1];
  const float2 a2L = pmul(vL[RBMOD], prcp(vL[RDENS])), a2R = pmul(vR[RBMOD], prcp(vR[RDENS]));
  const float2 cfL = make_float2(sqrtf(a2L.x), sqrtf(a2L.y)), cfR = make_float2(sqrtf(a2R.x), sqrtf(a2R.y));
  const float2 mL = psub(uL, cfL), mR = psub(uR, cfR), pL = padd(uL, cfL), pR = padd(uR, cfR);
  const float2 sL = make_float2(kmin(-tiny, kmin(mL.x, mR.x)), kmin(-tiny, kmin(mL.y, mR.y)));
  const float2 sR = make_float2(kmax(tiny, kmax(pL.x, pR.x)), kmax(tiny, kmax(pL.y, pR.y)));
  float2 UL[5], UR[5], FL[5], FR[5];
  Prim2ConsFlux2<DIR1>(vL, UL, FL);
  Prim2ConsFlux2<DIR1>(vR, UR, FR);
  if constexpr (RIEMANN == HLL) {
    const float2 sRmsLi = prcp(psub(sR, sL)), sRsL = pmul(sR, sL);
#pragma unroll
    for (int v = 0; v < 5; v++)
      flux[v] = pmul(sRmsLi, pfma(sRsL, psub(UR[v], UL[v]), psub(pmul(sR, FL[v]), pmul(sL, FR[v]))));
  } else {
    const float2 dL = psub(sL, uL), dR = psub(sR, uR);
    const float2 rdL = pmul(vL[RDENS], dL), rdR = pmul(vR[RDENS], dR);
    float2 ustar = psub(pfma(UL[CMOM0 + DIR1], dL, psub(vR[RPRES], vL[RPRES])), pmul(UR[CMOM0 + DIR1], dR));
    ustar = pmul(ustar, prcp(psub(rdL, rdR)));
    const float2 pstar = pmul(p2(0.5f), padd(padd(vL[RPRES], vR[RPRES]),
                                             pfma(rdL, psub(ustar, uL), pmul(rdR, psub(ustar, uR)))));
    const float2 pu = pmul(pstar, ustar);
    auto hllc_state = [&](float2 S, const float2 *U, float2 Pu, float2 *Us) {
      const float2 susi = prcp(padd(psub(S, ustar), p2(tiny)));
      Us[CDENS] = pmul(susi, psub(pmul(S, U[CDENS]), U[CMOM0 + DIR1]));
      Us[CMOM0 + DIR1] = pmul(Us[CDENS], ustar);
      const float2 ratio = pmul(Us[CDENS], prcp(U[CDENS]));
      Us[CMOM0 + DIR2] = pmul(U[CMOM0 + DIR2], ratio);
      Us[CMOM0 + DIR3] = pmul(U[CMOM0 + DIR3], ratio);
      Us[CENER] = pfma(U[CENER], ratio, pmul(susi, psub(pu, Pu)));
    };
    float2 UsL[5], UsR[5];
    hllc_state(sL, UL, pmul(vL[RPRES], uL), UsL);
    hllc_state(sR, UR, pmul(vR[RPRES], uR), UsR);
    const float2 sg = make_float2(copysignf(1.f, ustar.x), copysignf(1.f, ustar.y));
    const float2 biasL = make_float2(-kmin(-tiny, sg.x), -kmin(-tiny, sg.y));
    const float2 biasR = make_float2(kmax(tiny, sg.x), kmax(tiny, sg.y));
#pragma unroll
    for (int v = 0; v < 5; v++)
      flux[v] = pfma(biasR, pfma(sL, psub(UsL[v], UL[v]), FL[v]), pmul(biasL, pfma(sR, psub(UsR[v], UR[v]), FR[v])));
  }
}

// ---------------------------------------------------------------------------
// Ideal-gas EOS (singularity::IdealGas as used at equation_of_state.hpp:40-64).
struct EosParams {
  double gm1;  // gamma - 1
  double cv;   // gamma * kB / Abar
};

// ener mode: rho, sie -> T, P, bulk modulus
template <typename R>
__device__ __forceinline__ void EosEner(const EosParams &e, R rho, R sie, R &temp, R &pres,
                                        R &bmod) {
  const R gm1 = R(e.gm1);
  pres = kmax(R(0), gm1 * rho * sie);
  temp = kmax(R(0), kdiv(sie, R(e.cv)));
  bmod = kmax(R(0), (gm1 + R(1)) * gm1 * rho * sie);
}

// Cons2Prim (primconsflux.hpp:76-98) + ener-mode EOS on one cell.  E is passed
// in double so the FP32 path recovers e_int = E - e_kin - e_mag in FP64.
template <bool MHD, typename R>
__device__ __forceinline__ void Cons2PrimEos(const EosParams &eos, R dens, R m0, R m1, R m2,
                                             double ener, const R *B, R *V) {
  const R idens = kdiv(R(1.0), dens);
  V[RDENS] = dens;
  V[RVEL0] = idens * m0;
  V[RVEL1] = idens * m1;
  V[RVEL2] = idens * m2;
  R sie;
  if constexpr (sizeof(R) == sizeof(double)) {
    R ekin = R(0), emag = R(0);
    ekin += V[RVEL0] * V[RVEL0];
    ekin += V[RVEL1] * V[RVEL1];
    ekin += V[RVEL2] * V[RVEL2];
    if constexpr (MHD) {
      for (int d = 0; d < 3; d++) emag += B[d] * B[d];
    }
    ekin *= R(0.5) * dens;
    emag *= R(0.5);
    const R eint = R(ener) - ekin - emag;
    sie = idens * eint;
  } else {
    // FP32 storage: kinetic and magnetic energies and the subtraction in FP64
    const double dd = double(dens);
    // 1/rho in FP64 from the FP32 reciprocal and one Newton-Raphson step,
    // x1 = x0 + x0 (1 - rho x0): the relative error becomes about the square
    // of the FP32 one (< 1e-13), with no FP64 division.
    const double r0 = double(R(1) / dens);
    const double id = fma(r0, fma(-dd, r0, 1.0), r0);
    const double u0 = id * double(m0), u1 = id * double(m1), u2 = id * double(m2);
    double ekin = (u0 * u0 + u1 * u1 + u2 * u2) * (0.5 * dd);
    double emag = 0.0;
    if constexpr (MHD) {
      for (int d = 0; d < 3; d++) emag += double(B[d]) * double(B[d]);
      emag *= 0.5;
    }
    sie = R(id * (ener - ekin - emag));
  }
  V[REINT] = sie;
  R temp;
  EosEner(eos, dens, sie, temp, V[RPRES], V[RBMOD]);
  if constexpr (MHD) {
    V[RMAGC0] = B[0];
    V[RMAGC0 + 1] = B[1];
    V[RMAGC0 + 2] = B[2];
  }
}

// splitmix64 (Steele, Lea & Flood 2014) as a counter-based generator.
__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ double kh_uniform(uint64_t seed, uint64_t gidx, int comp) {
  const uint64_t h = splitmix64(splitmix64(seed) ^ (gidx * 2u + uint64_t(comp)));
  return double(h >> 11) * 0x1.0p-53;
}

}  // namespace kmy

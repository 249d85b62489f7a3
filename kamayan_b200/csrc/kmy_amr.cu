// kmy_amr.cu -- adaptive mesh refinement: boundary exchange across levels,
// flux correction at fine/coarse faces, Loehner tagging, and the remesh (tree
// update on the host, data remap on the device).
//
// Semantics (Parthenon's block tree and exchange are un-vendored and restated;
// the operators are kamayan's):
//   RestrictAverage            refinement_operations.hpp:56-120
//   ProlongateSharedGeneral    refinement_operations.hpp:123-264 (minmod)
//   GradMinMod                 refinement_operations.hpp:44-50
//   AMRLoehner::operator()     grid_refinement.cpp:30-152
//   flux correction task       kamayan_driver.cpp:206-207
//   tagging before exchange    kamayan_driver.cpp:178-181, :150-151
//
// The value of a cell at level L and global index G is the best
// representation the mesh has there: the cell of the level-L leaf that holds
// it, the volume-weighted restriction of the finer leaves covering it, or the
// minmod prolongation from level L-1.  Ghost cells, cells remapped by a remesh
// and the coarse stencils of a prolongation all take that value.  With 2:1
// balance (corners included) the recursion stays within a few levels; it is
// unrolled to a fixed depth so the stack size is known at compile time, and a
// deeper request sets an error flag instead of recursing.
//
// The unit is compiled without FMA contraction, so each expression rounds as
// written and tag decisions match a CPU evaluation of the same expressions.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <vector>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

namespace kmy {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxDepth = 12;               // unrolled depth of the level value
// CTAs per SM the level-value kernels keep resident.  The recursive
// evaluation otherwise takes all 255 registers (one CTA per SM); bounded, its
// rarely entered deep frames spill instead.
constexpr int kLvBlocks = 4;
constexpr long long kMaxTable = 1ll << 26;  // level-table entries over all levels

unsigned nblk(long long n) { return unsigned((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ long long cidx(const MeshDesc &m, int k, int j, int i) {
  return ((long long)k * m.np[1] + j) * m.np[0] + i;
}
__device__ __forceinline__ long long fidx(const MeshDesc &m, int k, int j, int i) {
  return ((long long)k * m.nf[1] + j) * m.nf[0] + i;
}

// Physical boundary map of a global index on an N-cell axis.
__device__ __forceinline__ int amr_map(int G, int N, int bc, bool &flip) {
  if (G >= 0 && G < N) return G;
  if (bc == BC_PERIODIC) return ((G % N) + N) % N;
  if (bc == BC_OUTFLOW) return G < 0 ? 0 : N - 1;
  flip = !flip;
  return G < 0 ? -G - 1 : 2 * N - G - 1;
}

// Leaf id at block position bx of level L, -1 when finer leaves cover it,
// -2 when a coarser leaf does (or L is outside the tables).
__device__ __forceinline__ int table_at(const MeshDesc &m, int L, const int bx[3]) {
  if (L < 0 || L >= m.nlev) return -2;
  return m.tabs[m.tab_off[L] + ((long long)bx[2] * m.tab_dim[L][1] + bx[1]) * m.tab_dim[L][0] + bx[0]];
}

// One stored variable over [nb][P]: FP64, or FP32 with an optional low word.
struct Field {
  const void *p;
  const float *lo;
  int f32;
};
__device__ __forceinline__ double fetch(const Field &f, long long n) {
  if (f.f32) {
    double v = double(static_cast<const float *>(f.p)[n]);
    if (f.lo) v += double(f.lo[n]);
    return v;
  }
  return static_cast<const double *>(f.p)[n];
}

// RestrictAverage over the 2^d children, index (ok*4 + oj*2 + oi); the sums
// keep the operator's pairing.
__device__ __forceinline__ double restrict8(const double t[8], const double v[8]) {
  const double tvol = ((v[0] + v[2]) + (v[1] + v[3])) + ((v[4] + v[6]) + (v[5] + v[7]));
  return tvol > 0.0 ? (((t[0] + t[2]) + (t[1] + t[3])) + ((t[4] + t[6]) + (t[5] + t[7]))) / tvol : 0.0;
}

// GradMinMod with SIGN(x) = x < 0 ? -1 : 1
__device__ __forceinline__ double grad_minmod(double fc, double fm, double fp, double dxm, double dxp) {
  const double gxm = (fc - fm) / dxm;
  const double gxp = (fp - fc) / dxp;
  const double sm = gxm < 0 ? -1.0 : 1.0, sp = gxp < 0 ? -1.0 : 1.0;
  const double agm = fabs(gxm), agp = fabs(gxp);
  return 0.5 * (sm + sp) * ((agp < agm) ? agp : agm);
}

template <int D>
__device__ __noinline__ double level_value(const MeshDesc &m, int L, int G0, int G1, int G2, const Field &f,
                                           int flipdim, int *err);

// level_value with its common case inline: a position that holds a leaf at
// level L is fetched directly, and only restriction or prolongation enters the
// recursive (register-heavy, non-inlined) evaluation.  Same arithmetic.
template <int D>
__device__ __forceinline__ double level_value_at(const MeshDesc &m, int L, int G0, int G1, int G2, const Field &f,
                                                 int flipdim, int *err) {
  const int G[3] = {G0, G1, G2};
  int M[3] = {0, 0, 0};
  bool flip[3] = {false, false, false};
  for (int d = 0; d < m.ndim; d++) M[d] = amr_map(G[d], m.mesh_nx[d] << L, m.bc[d][G[d] < 0 ? 0 : 1], flip[d]);
  int bx[3];
  for (int d = 0; d < 3; d++) bx[d] = M[d] / m.nx[d];
  const int e = table_at(m, L, bx);
  if (e >= 0) {
    const double sgn = (flipdim >= 0 && flip[flipdim]) ? -1.0 : 1.0;
    return sgn * fetch(f, (long long)e * m.P + cidx(m, M[2] - bx[2] * m.nx[2] + m.g[2],
                                                    M[1] - bx[1] * m.nx[1] + m.g[1],
                                                    M[0] - bx[0] * m.nx[0] + m.g[0]));
  }
  return level_value<D>(m, L, G0, G1, G2, f, flipdim, err);
}

// Value of field f at level L, global cell G; flipdim is the vector component
// the field carries (its sign flips across reflecting boundaries) or -1.
template <int D>
__device__ __noinline__ double level_value(const MeshDesc &m, int L, int G0, int G1, int G2, const Field &f,
                                           int flipdim, int *err) {
  const int G[3] = {G0, G1, G2};
  int M[3] = {0, 0, 0};
  bool flip[3] = {false, false, false};
  for (int d = 0; d < m.ndim; d++) {
    const int N = m.mesh_nx[d] << L;
    M[d] = amr_map(G[d], N, m.bc[d][G[d] < 0 ? 0 : 1], flip[d]);
  }
  const double sgn = (flipdim >= 0 && flip[flipdim]) ? -1.0 : 1.0;
  int bx[3];
  for (int d = 0; d < 3; d++) bx[d] = M[d] / m.nx[d];
  const int e = table_at(m, L, bx);
  if (e >= 0)
    return sgn * fetch(f, (long long)e * m.P + cidx(m, M[2] - bx[2] * m.nx[2] + m.g[2],
                                                    M[1] - bx[1] * m.nx[1] + m.g[1],
                                                    M[0] - bx[0] * m.nx[0] + m.g[0]));
  if constexpr (D == 0) {
    *err = 1;
    return 0.0;
  } else {
    const int nd = m.ndim;
    if (e == -1) {  // covered by finer leaves: restrict from level L+1
      double t[8] = {0, 0, 0, 0, 0, 0, 0, 0}, v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      double vol = 1.0;
      for (int d = 0; d < 3; d++) vol *= d < nd ? m.dx[d] / double(1 << (L + 1)) : m.dx[d];
      for (int ok = 0; ok < 1 + (nd > 2); ok++)
        for (int oj = 0; oj < 1 + (nd > 1); oj++)
          for (int oi = 0; oi < 2; oi++) {
            const int q = ok * 4 + oj * 2 + oi;
            v[q] = vol;
            t[q] = vol * level_value_at<D - 1>(m, L + 1, 2 * M[0] + oi, nd > 1 ? 2 * M[1] + oj : 0,
                                            nd > 2 ? 2 * M[2] + ok : 0, f, flipdim, err);
          }
      return sgn * restrict8(t, v);
    }
    if (L == 0) {  // a level-0 position always has a leaf at or below it
      *err = 2;
      return 0.0;
    }
    // covered by a coarser leaf: prolongate from level L-1
    int Mc[3] = {0, 0, 0}, o[3] = {0, 0, 0};
    for (int d = 0; d < nd; d++) {
      Mc[d] = M[d] >> 1;
      o[d] = M[d] & 1;
    }
    const double fc = level_value_at<D - 1>(m, L - 1, Mc[0], Mc[1], Mc[2], f, flipdim, err);
    double gq[3] = {0, 0, 0}, dfm[3] = {0, 0, 0}, dfp[3] = {0, 0, 0};
    for (int d = 0; d < nd; d++) {
      const double dxc = m.dx[d] / double(1 << (L - 1)), dxf = m.dx[d] / double(1 << L);
      const double x0 = m.xmin[d];
      int Gm[3] = {Mc[0], Mc[1], Mc[2]}, Gp[3] = {Mc[0], Mc[1], Mc[2]};
      Gm[d] -= 1;
      Gp[d] += 1;
      const double fm = level_value_at<D - 1>(m, L - 1, Gm[0], Gm[1], Gm[2], f, flipdim, err);
      const double fp = level_value_at<D - 1>(m, L - 1, Gp[0], Gp[1], Gp[2], f, flipdim, err);
      const double xm = x0 + (double(Mc[d] - 1) + 0.5) * dxc;
      const double xc = x0 + (double(Mc[d]) + 0.5) * dxc;
      const double xp = x0 + (double(Mc[d] + 1) + 0.5) * dxc;
      const double dxm = xc - xm, dxp = xp - xc;
      dfm[d] = xc - (x0 + (double(2 * Mc[d]) + 0.5) * dxf);
      dfp[d] = (x0 + (double(2 * Mc[d] + 1) + 0.5) * dxf) - xc;
      gq[d] = grad_minmod(fc, fm, fp, dxm, dxp);
    }
    const double g1 = gq[0], g2 = gq[1], g3 = gq[2];
    const double d1m = dfm[0], d1p = dfp[0], d2m = dfm[1], d2p = dfp[1], d3m = dfm[2], d3p = dfp[2];
    double val;
    switch (o[0] + 2 * o[1] + 4 * o[2]) {
      case 0: val = fc - (g1 * d1m + g2 * d2m + g3 * d3m); break;
      case 1: val = fc + (g1 * d1p - g2 * d2m - g3 * d3m); break;
      case 2: val = fc - (g1 * d1m - g2 * d2p + g3 * d3m); break;
      case 3: val = fc + (g1 * d1p + g2 * d2p - g3 * d3m); break;
      case 4: val = fc - (g1 * d1m + g2 * d2m - g3 * d3p); break;
      case 5: val = fc + (g1 * d1p - g2 * d2m + g3 * d3p); break;
      case 6: val = fc - (g1 * d1m - g2 * d2p - g3 * d3p); break;
      default: val = fc + (g1 * d1p + g2 * d2p + g3 * d3p); break;
    }
    return sgn * val;
  }
}

// Face arrays [3][nb][Pf] of one container.
struct FaceField {
  const void *p;
  long long NF;  // nb * Pf
  int f32;
};
__device__ __forceinline__ double ffetch(const FaceField &f, int e, long long n) {
  const long long i = e * f.NF + n;
  return f.f32 ? double(static_cast<const float *>(f.p)[i]) : static_cast<const double *>(f.p)[i];
}

// Global index along axis d of a face of component e at level L: along e
// out-of-range faces clamp to the boundary face (or wrap when periodic),
// across e the cell map applies; 0 in inactive dimensions.
__device__ __forceinline__ int face_axis_map(const MeshDesc &m, int d, int e, int L, int Gd) {
  if (d >= m.ndim) return 0;
  const int N = m.mesh_nx[d] << L;
  if (d == e) {
    if (Gd >= 0 && Gd <= N) return Gd;
    if (m.bc[d][Gd < 0 ? 0 : 1] == BC_PERIODIC) return ((Gd % N) + N) % N;
    return Gd < 0 ? 0 : N;
  }
  bool fl = false;
  return amr_map(Gd, N, m.bc[d][Gd < 0 ? 0 : 1], fl);
}

// Small fixed-size vectors held in registers (selects instead of indexed
// local arrays) for the face recursion.
struct I3 {
  int v0, v1, v2;
  __device__ __forceinline__ int operator[](int d) const { return d == 0 ? v0 : d == 1 ? v1 : v2; }
  __device__ __forceinline__ void set(int d, int x) {
    if (d == 0) v0 = x;
    else if (d == 1) v1 = x;
    else v2 = x;
  }
};
struct R3 {
  double v0, v1, v2;
  __device__ __forceinline__ double operator[](int d) const { return d == 0 ? v0 : d == 1 ? v1 : v2; }
  __device__ __forceinline__ void set(int d, double x) {
    if (d == 0) v0 = x;
    else if (d == 1) v1 = x;
    else v2 = x;
  }
};

// Every face_value evaluation a thread may make before it gives up (the
// error flag is set and 0 returned), so a malformed tree cannot make a launch
// run away.
constexpr int kFaceBudget = 1 << 16;

// Value of face component e at level L, global face index G (face index along
// e, cell indices across).  Preference as for cells: the face of a level-L
// leaf (its low face, else the high face of the leaf below it along e), the
// area-weighted restriction of the finer leaves' faces on the same plane, or
// a prolongation from level L-1: faces on a coarse face plane by minmod in
// the plane (ProlongateSharedMinMod), faces inside a coarse cell by Toth & Roe
// (ProlongateInternalTothAndRoe, refinement_operations.hpp:270-398).
template <int D>
__device__ __noinline__ double face_value(const MeshDesc &m, int e, int L, int G0, int G1, int G2,
                                          const FaceField &f, int *err, int *calls) {
  if (++*calls > kFaceBudget) {
    *err = 3;
    return 0.0;
  }
  const I3 M{face_axis_map(m, 0, e, L, G0), face_axis_map(m, 1, e, L, G1), face_axis_map(m, 2, e, L, G2)};
  const bool act = e < m.ndim;
  const I3 bx{M.v0 / m.nx[0], M.v1 / m.nx[1], M.v2 / m.nx[2]};
  I3 bl = bx;
  const int NBe = act ? (m.nbx[e] << L) : 1;
  int ehi = -3, elo = -3;
  if (bx[e] < NBe) {
    const int q3[3] = {bx.v0, bx.v1, bx.v2};
    ehi = table_at(m, L, q3);
  }
  if (act && M[e] % m.nx[e] == 0 && M[e] > 0) {
    bl.set(e, bx[e] - 1);
    const int q3[3] = {bl.v0, bl.v1, bl.v2};
    elo = table_at(m, L, q3);
  }
  if (ehi >= 0 || elo >= 0) {
    const I3 q = ehi >= 0 ? bx : bl;
    int l0 = M.v0 - q.v0 * m.nx[0] + m.g[0], l1 = M.v1 - q.v1 * m.nx[1] + m.g[1], l2 = M.v2 - q.v2 * m.nx[2] + m.g[2];
    if (ehi < 0) {
      const int le = m.nx[e] + m.g[e];
      if (e == 0) l0 = le;
      else if (e == 1) l1 = le;
      else l2 = le;
    }
    return ffetch(f, e, (long long)(ehi >= 0 ? ehi : elo) * m.Pf + fidx(m, l2, l1, l0));
  }
  if constexpr (D == 0) {
    *err = 1;
    return 0.0;
  } else {
    const int nd = m.ndim;
    if (ehi == -1 || elo == -1) {  // finer leaves: restrict the fine faces on this plane
      double area = 1.0;
      for (int d = 0; d < 3; d++)
        if (d != e) area *= d < nd ? m.dx[d] / double(1 << (L + 1)) : m.dx[d];
      const int in0 = e != 0, in1 = e != 1 && nd > 1, in2 = e != 2 && nd > 2;
      // slots (ok*4 + oj*2 + oi); at most two offsets vary for a face
      double t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0;
      double w0 = 0, w1 = 0, w2 = 0, w3 = 0, w4 = 0, w5 = 0, w6 = 0, w7 = 0;
      for (int ok = 0; ok < 1 + in2; ok++)
        for (int oj = 0; oj < 1 + in1; oj++)
          for (int oi = 0; oi < 1 + in0; oi++) {
            const double val = area * face_value<D - 1>(m, e, L + 1, 2 * M.v0 + oi, nd > 1 ? 2 * M.v1 + oj : 0,
                                                        nd > 2 ? 2 * M.v2 + ok : 0, f, err, calls);
            switch (ok * 4 + oj * 2 + oi) {
              case 0: t0 = val; w0 = area; break;
              case 1: t1 = val; w1 = area; break;
              case 2: t2 = val; w2 = area; break;
              case 3: t3 = val; w3 = area; break;
              case 4: t4 = val; w4 = area; break;
              case 5: t5 = val; w5 = area; break;
              case 6: t6 = val; w6 = area; break;
              default: t7 = val; w7 = area; break;
            }
          }
      const double tvol = ((w0 + w2) + (w1 + w3)) + ((w4 + w6) + (w5 + w7));
      return tvol > 0.0 ? (((t0 + t2) + (t1 + t3)) + ((t4 + t6) + (t5 + t7))) / tvol : 0.0;
    }
    if (L == 0) {
      *err = 2;
      return 0.0;
    }
    if (!act || M[e] % 2 == 0) {  // shared face: minmod in the coarse face's plane
      I3 Mc{0, 0, 0}, o{0, 0, 0};
      for (int d = 0; d < nd; d++) {
        Mc.set(d, d == e ? M[d] / 2 : M[d] >> 1);
        o.set(d, d == e ? 0 : M[d] & 1);
      }
      const double fc = face_value<D - 1>(m, e, L - 1, Mc.v0, Mc.v1, Mc.v2, f, err, calls);
      R3 gq{0, 0, 0}, dfm{0, 0, 0}, dfp{0, 0, 0};
      for (int d = 0; d < nd; d++) {
        if (d == e) continue;
        const double dxc = m.dx[d] / double(1 << (L - 1)), dxf = m.dx[d] / double(1 << L);
        const double x0 = m.xmin[d];
        I3 Gm = Mc, Gp = Mc;
        Gm.set(d, Mc[d] - 1);
        Gp.set(d, Mc[d] + 1);
        const double fm = face_value<D - 1>(m, e, L - 1, Gm.v0, Gm.v1, Gm.v2, f, err, calls);
        const double fp = face_value<D - 1>(m, e, L - 1, Gp.v0, Gp.v1, Gp.v2, f, err, calls);
        const double xm = x0 + (double(Mc[d] - 1) + 0.5) * dxc;
        const double xc = x0 + (double(Mc[d]) + 0.5) * dxc;
        const double xp = x0 + (double(Mc[d] + 1) + 0.5) * dxc;
        dfm.set(d, xc - (x0 + (double(2 * Mc[d]) + 0.5) * dxf));
        dfp.set(d, (x0 + (double(2 * Mc[d] + 1) + 0.5) * dxf) - xc);
        gq.set(d, grad_minmod(fc, fm, fp, xc - xm, xp - xc));
      }
      const double g1 = gq.v0, g2 = gq.v1, g3 = gq.v2;
      const double d1m = dfm.v0, d1p = dfp.v0, d2m = dfm.v1, d2p = dfp.v1, d3m = dfm.v2, d3p = dfp.v2;
      switch (o.v0 + 2 * o.v1 + 4 * o.v2) {
        case 0: return fc - (g1 * d1m + g2 * d2m + g3 * d3m);
        case 1: return fc + (g1 * d1p - g2 * d2m - g3 * d3m);
        case 2: return fc - (g1 * d1m - g2 * d2p + g3 * d3m);
        case 3: return fc + (g1 * d1p + g2 * d2p - g3 * d3m);
        case 4: return fc - (g1 * d1m + g2 * d2m - g3 * d3p);
        case 5: return fc + (g1 * d1p - g2 * d2m + g3 * d3p);
        case 6: return fc - (g1 * d1m - g2 * d2p - g3 * d3p);
        default: return fc + (g1 * d1p + g2 * d2p + g3 * d3p);
      }
    }
    // internal face (odd along e): Toth & Roe from the level-L faces on the
    // coarse cell's boundary; offsets oi along a0 = e, oj along a1, ok along
    // a2, collapsed in inactive dimensions (where the operator's second write,
    // offset 1, is the one that stays)
    const int a0 = e, a1 = (e + 1) % 3, a2 = (e + 2) % 3;
    const I3 f0{nd > 0 ? 2 * (M.v0 >> 1) : 0, nd > 1 ? 2 * (M.v1 >> 1) : 0, nd > 2 ? 2 * (M.v2 >> 1) : 0};
    const I3 act3{nd > 0 ? 1 : 0, nd > 1 ? 1 : 0, nd > 2 ? 1 : 0};
    auto fine = [&](int eidx, int ok, int oj, int oi) {
      I3 P = f0;
      P.set(a0, P[a0] + oi * act3[a0]);
      P.set(a1, P[a1] + oj * act3[a1]);
      P.set(a2, P[a2] + ok * act3[a2]);
      return face_value<D - 1>(m, (e + eidx) % 3, L, P.v0, P.v1, P.v2, f, err, calls);
    };
    auto sg = [](int off) { return off == 0 ? -1.0 : 1.0; };
    double Uxx = 0.0, Vxyz = 0.0, Wxyz = 0.0;
    for (int vv = 0; vv < 2; vv++)
      for (int u = 0; u <= 2; u += 2)
        for (int t = 0; t < 2; t++) {
          const double fine2 = fine(1, vv, u, t);
          const double fine3 = fine(2, u, vv, t);
          Uxx += sg(t) * sg(u) * (fine2 + fine3);
          Vxyz += sg(t) * sg(u) * sg(vv) * fine2;
          Wxyz += sg(t) * sg(u) * sg(vv) * fine3;
        }
    Uxx *= 0.125;
    const double c0 = nd > 0 ? m.dx[0] / double(1 << (L - 1)) : m.dx[0];
    const double c1 = nd > 1 ? m.dx[1] / double(1 << (L - 1)) : m.dx[1];
    const double c2 = nd > 2 ? m.dx[2] / double(1 << (L - 1)) : m.dx[2];
    const double dx2 = c0 * c0, dy2 = c1 * c1, dz2 = c2 * c2;
    Vxyz *= 0.125 * dz2 / (dx2 + dz2);
    Wxyz *= 0.125 * dy2 / (dx2 + dy2);
    const int ok = act3[a2] ? M[a2] - f0[a2] : 1;
    const int oj = act3[a1] ? M[a1] - f0[a1] : 1;
    return 0.5 * (fine(0, ok, oj, 0) + fine(0, ok, oj, 2)) + Uxx + sg(ok) * Vxyz + sg(oj) * Wxyz;
  }
}

template <typename S>
__device__ __forceinline__ void store_value(S *arr, float *lo, long long n, double v) {
  if constexpr (sizeof(S) == 4) {
    const float hi = float(v);
    arr[n] = hi;
    if (lo) lo[n] = float(v - double(hi));
  } else {
    arr[n] = v;
  }
}

// ---------------------------------------------------------------------------
// Ghost plan.  The ghost cells whose position is not a leaf at their level
// (fine/coarse boundaries) are listed once per table upload with the cells
// their restriction or prolongation reads, so a ghost fill reads them
// directly instead of walking the tree per variable and stage.  A source
// that is no leaf either but is itself one restriction or prolongation of
// leaves (a prolongation's coarse neighbour where the levels change again,
// near block corners) becomes an inner entry: its value goes to a scratch
// slot first and the outer entry reads it there.  Anything deeper keeps the
// recursive evaluation.  The arithmetic is level_value's, term for term.
struct GhostPlan {
  long long dst;      // outer entry: ghost cell, offset in [nb][P]; inner entry: scratch slot
  long long src[8];   // restriction: the 2^d children (index ok*4 + oj*2 + oi);
                      // prolongation: the coarse cell, then its - / + neighbours per axis;
                      // >= 0 a leaf cell's offset, < 0 scratch slot -src - 1
  int kind;           // 1 restriction, 2 prolongation, 3 recursive evaluation at fill time
  int flips;          // bits 0-2: the ghost position's mirrored axes (0 for inner entries);
                      // prolongation: bits 3(k+1)+d those of source k
  int L;              // level of the position
  int M[3];           // its mapped position at L (kind 3: the unmapped global position)
};

// Mapped position M, mirrored axes fl and table entry of global position P
// at level L.
__device__ __forceinline__ int plan_map(const MeshDesc &m, int L, const int P[3], int M[3], int &fl) {
  bool flip[3] = {false, false, false};
  M[0] = M[1] = M[2] = 0;
  for (int d = 0; d < m.ndim; d++) M[d] = amr_map(P[d], m.mesh_nx[d] << L, m.bc[d][P[d] < 0 ? 0 : 1], flip[d]);
  int bx[3];
  for (int d = 0; d < 3; d++) bx[d] = M[d] / m.nx[d];
  fl = (flip[0] ? 1 : 0) | (flip[1] ? 2 : 0) | (flip[2] ? 4 : 0);
  return table_at(m, L, bx);
}

// Offset of the leaf holding global position P at level L, or -1 when no
// leaf does; fl gets the axes the boundary map mirrored.
__device__ __forceinline__ long long plan_leaf(const MeshDesc &m, int L, const int P[3], int &fl) {
  int M[3];
  const int e = plan_map(m, L, P, M, fl);
  if (e < 0) return -1;
  int bx[3];
  for (int d = 0; d < 3; d++) bx[d] = M[d] / m.nx[d];
  return (long long)e * m.P + cidx(m, M[2] - bx[2] * m.nx[2] + m.g[2], M[1] - bx[1] * m.nx[1] + m.g[1],
                                   M[0] - bx[0] * m.nx[0] + m.g[0]);
}

// Level and global position P of source k of a restriction (kind 1) or a
// prolongation (kind 2) at mapped position M of level L.
__device__ __forceinline__ int plan_source(const MeshDesc &m, int kind, int L, const int M[3], int k, int P[3]) {
  const int nd = m.ndim;
  if (kind == 1) {
    P[0] = 2 * M[0] + (k & 1);
    P[1] = nd > 1 ? 2 * M[1] + ((k >> 1) & 1) : 0;
    P[2] = nd > 2 ? 2 * M[2] + ((k >> 2) & 1) : 0;
    return L + 1;
  }
  for (int d = 0; d < 3; d++) P[d] = d < nd ? M[d] >> 1 : 0;
  if (k > 0) P[(k - 1) >> 1] += (k & 1) ? -1 : 1;  // k = 1 + 2d: the - neighbour, 2 + 2d: the +
  return L - 1;
}

// Kind and sources of mapped position M at level L, whose table entry e is
// no leaf: a leaf source gets its offset, any other -1 and its bit in the
// returned mask.  kind 3 when neither restriction nor prolongation applies
// (a level-0 position without a leaf, which the recursion reports).
__device__ __forceinline__ unsigned plan_node(const MeshDesc &m, int L, const int M[3], int e, GhostPlan &g) {
  g.L = L;
  for (int d = 0; d < 3; d++) g.M[d] = M[d];
  for (int q = 0; q < 8; q++) g.src[q] = 0;
  g.flips = 0;
  if (e == -1) g.kind = 1;
  else if (L > 0) g.kind = 2;
  else {
    g.kind = 3;
    return 0;
  }
  const int ns = g.kind == 1 ? 1 << m.ndim : 1 + 2 * m.ndim;
  unsigned miss = 0;
  for (int k = 0; k < ns; k++) {
    int P[3], fl;
    const int Ls = plan_source(m, g.kind, L, M, k, P);
    g.src[k] = plan_leaf(m, Ls, P, fl);
    if (g.kind == 2) g.flips |= fl << (3 * (k + 1));
    if (g.src[k] < 0) miss |= 1u << k;
  }
  return miss;
}

// Inner entry for source k of g, which is no leaf: true when it is one
// restriction or prolongation of leaves.
__device__ __forceinline__ bool plan_inner(const MeshDesc &m, const GhostPlan &g, int k, GhostPlan &in) {
  int P[3], M[3], fl;
  const int Ls = plan_source(m, g.kind, g.L, g.M, k, P);
  const int e = plan_map(m, Ls, P, M, fl);
  if (e >= 0) return false;
  return plan_node(m, Ls, M, e, in) == 0 && in.kind != 3;
}

// Same-level ghost copies (the common case): the ghost cell, the leaf cell
// holding its position, and the axes the boundary map mirrored.
struct GhostCopy {
  long long dst, src;
  int flips;
};

// Padded cell t: 0 when interior; 1 when its position holds a leaf at its
// level (cp: the copy); 2 otherwise (g: the outer entry; miss: the sources
// that need an inner entry; kind 3 when one of them is deeper still).
__device__ __forceinline__ int plan_entry(const MeshDesc &m, unsigned t, GhostPlan &g, unsigned &miss,
                                          GhostCopy &cp) {
  const unsigned P = unsigned(m.P);
  const int b = int(t / P);
  unsigned r = t - unsigned(b) * P;
  const int loc[3] = {int(r % unsigned(m.np[0])), int((r / unsigned(m.np[0])) % unsigned(m.np[1])),
                      int(r / (unsigned(m.np[0]) * unsigned(m.np[1])))};
  bool interior = true;
  for (int d = 0; d < 3; d++)
    if (loc[d] < m.g[d] || loc[d] >= m.g[d] + m.nx[d]) interior = false;
  if (interior) return 0;
  const int L = m.blev[b];
  int G[3], M[3], ftop;
  for (int d = 0; d < 3; d++) G[d] = m.bloc[3 * b + d] * m.nx[d] + (loc[d] - m.g[d]);
  const int e = plan_map(m, L, G, M, ftop);
  const long long dst = (long long)b * m.P + cidx(m, loc[2], loc[1], loc[0]);
  if (e >= 0) {
    int bx[3];
    for (int d = 0; d < 3; d++) bx[d] = M[d] / m.nx[d];
    cp.dst = dst;
    cp.src = (long long)e * m.P + cidx(m, M[2] - bx[2] * m.nx[2] + m.g[2], M[1] - bx[1] * m.nx[1] + m.g[1],
                                       M[0] - bx[0] * m.nx[0] + m.g[0]);
    cp.flips = ftop;
    return 1;
  }
  miss = plan_node(m, L, M, e, g);
  g.dst = dst;
  g.flips |= ftop;
  for (int k = 0; k < 8 && g.kind != 3; k++) {
    GhostPlan in;
    if (((miss >> k) & 1) && !plan_inner(m, g, k, in)) g.kind = 3;
  }
  if (g.kind == 3) {
    miss = 0;
    for (int d = 0; d < 3; d++) g.M[d] = G[d];
  }
  return 2;
}

// count[0] counts the outer entries read directly, count[1] the recursive
// ones, count[2] the inner entries and count[3] the copies.  The fill pass
// stores the plan entries at [0, n0), [n0, n0 + n1) and [n0 + n1, ...), so a
// warp of the direct fill never waits on a recursion, and the copies apart.
__global__ void k_amr_plan(const __grid_constant__ MeshDesc m, GhostPlan *plan, GhostCopy *copies, int *count,
                           int n0, int n1) {
  const unsigned per = unsigned(m.nb) * unsigned(m.P);
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= per) return;
  GhostPlan g;
  GhostCopy cp;
  unsigned miss = 0;
  const int what = plan_entry(m, t, g, miss, cp);
  if (what == 0) return;
  if (what == 1) {
    const int q = atomicAdd(count + 3, 1);
    if (copies) copies[q] = cp;
    return;
  }
  if (g.kind == 3) {
    const int q = atomicAdd(count + 1, 1);
    if (plan) plan[n0 + q] = g;
    return;
  }
  int slot = miss ? atomicAdd(count + 2, __popc(miss)) : 0;
  if (plan) {
    for (int k = 0; k < 8; k++) {
      if (!((miss >> k) & 1)) continue;
      GhostPlan in;
      plan_inner(m, g, k, in);
      in.dst = slot;
      plan[n0 + n1 + slot] = in;
      g.src[k] = -1 - (long long)slot;
      slot++;
    }
  }
  const int q = atomicAdd(count, 1);
  if (plan) plan[q] = g;
}

// The variable v of the fill kernels (blockIdx.y: the ncc conserved
// variables, then the NPRIM primitives): its array, vector component (-1:
// scalar) and, for FP32 energy, low words.
template <typename S>
struct FillVar {
  S *arr;
  float *lo;
  int fd;
  __device__ __forceinline__ FillVar(const MeshDesc &m, int v, S *cc, float *clo, S *prim, int ncc) {
    const long long NP = (long long)m.nb * m.P;
    const bool is_cc = v < ncc;
    arr = is_cc ? cc + v * NP : prim + (v - ncc) * NP;
    fd = is_cc ? ((v >= CMOM0 && v <= CMOM2) ? v - CMOM0 : (v >= CMAGC0 ? v - CMAGC0 : -1))
               : (v - ncc <= PVEL2 ? v - ncc : -1);
    lo = (sizeof(S) == 4 && is_cc && v == CENER) ? clo : nullptr;
  }
};

// The same-level ghost copies: a copy of the leaf cell, mirrored components
// negated across a reflecting boundary; one thread per (copy, variable).
// Reads interior cells only.
template <typename S>
__global__ void k_amr_fill_copy(const __grid_constant__ MeshDesc m, const GhostCopy *copies, int n, S *cc,
                                float *lo, S *prim, int ncc) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const FillVar<S> fv(m, blockIdx.y, cc, lo, prim, ncc);
  const GhostCopy cp = copies[q];
  S val = fv.arr[cp.src];
  if (fv.fd >= 0 && ((cp.flips >> fv.fd) & 1)) val = -val;
  fv.arr[cp.dst] = val;
  if constexpr (sizeof(S) == 4) {
    if (fv.lo) fv.lo[cp.dst] = fv.lo[cp.src];
  }
}

// The plan's recursive entries [q0, q0 + n): level_value at the ghost
// position, one thread per (entry, variable).
template <typename S>
__global__ void __launch_bounds__(kThreads, kLvBlocks) k_amr_fill_plan_deep(const __grid_constant__ MeshDesc m,
                                                                            const GhostPlan *plan, int q0, int n,
                                                                            S *cc, float *lo, S *prim, int ncc,
                                                                            int *err) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const FillVar<S> fv(m, blockIdx.y, cc, lo, prim, ncc);
  const GhostPlan &g = plan[q0 + q];
  const Field f{fv.arr, fv.lo, sizeof(S) == 4};
  store_value<S>(fv.arr, fv.lo, g.dst, level_value_at<kMaxDepth>(m, g.L, g.M[0], g.M[1], g.M[2], f, fv.fd, err));
}

// Value of a restriction (kind 1) or prolongation (kind 2) entry for field f
// (vector component fd); scr holds this variable's scratch slots.
__device__ __forceinline__ double plan_value(const MeshDesc &m, const GhostPlan &g, const Field &f, int fd,
                                             const double *scr) {
  const int L = g.L, nd = m.ndim;
  auto src = [&](int k) {
    const long long s = g.src[k];
    return s >= 0 ? fetch(f, s) : scr[-s - 1];
  };
  auto sgn = [&](int k) { return (fd >= 0 && ((g.flips >> (3 * k + fd)) & 1)) ? -1.0 : 1.0; };
  if (g.kind == 1) {
    double t[8] = {0, 0, 0, 0, 0, 0, 0, 0}, vv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double vol = 1.0;
    for (int d = 0; d < 3; d++) vol *= d < nd ? m.dx[d] / double(1 << (L + 1)) : m.dx[d];
    for (int ok = 0; ok < 1 + (nd > 2); ok++)
      for (int oj = 0; oj < 1 + (nd > 1); oj++)
        for (int oi = 0; oi < 2; oi++) {
          const int c = ok * 4 + oj * 2 + oi;
          vv[c] = vol;
          t[c] = vol * src(c);
        }
    return sgn(0) * restrict8(t, vv);
  }
  int Mc[3] = {0, 0, 0}, o[3] = {0, 0, 0};
  for (int d = 0; d < nd; d++) {
    Mc[d] = g.M[d] >> 1;
    o[d] = g.M[d] & 1;
  }
  const double fc = sgn(1) * src(0);
  double gq[3] = {0, 0, 0}, dfm[3] = {0, 0, 0}, dfp[3] = {0, 0, 0};
  for (int d = 0; d < nd; d++) {
    const double dxc = m.dx[d] / double(1 << (L - 1)), dxf = m.dx[d] / double(1 << L);
    const double x0 = m.xmin[d];
    const double fm = sgn(2 + 2 * d) * src(1 + 2 * d);
    const double fp = sgn(3 + 2 * d) * src(2 + 2 * d);
    const double xm = x0 + (double(Mc[d] - 1) + 0.5) * dxc;
    const double xc = x0 + (double(Mc[d]) + 0.5) * dxc;
    const double xp = x0 + (double(Mc[d] + 1) + 0.5) * dxc;
    const double dxm = xc - xm, dxp = xp - xc;
    dfm[d] = xc - (x0 + (double(2 * Mc[d]) + 0.5) * dxf);
    dfp[d] = (x0 + (double(2 * Mc[d] + 1) + 0.5) * dxf) - xc;
    gq[d] = grad_minmod(fc, fm, fp, dxm, dxp);
  }
  const double g1 = gq[0], g2 = gq[1], g3 = gq[2];
  const double d1m = dfm[0], d1p = dfp[0], d2m = dfm[1], d2p = dfp[1], d3m = dfm[2], d3p = dfp[2];
  double pv;
  switch (o[0] + 2 * o[1] + 4 * o[2]) {
    case 0: pv = fc - (g1 * d1m + g2 * d2m + g3 * d3m); break;
    case 1: pv = fc + (g1 * d1p - g2 * d2m - g3 * d3m); break;
    case 2: pv = fc - (g1 * d1m - g2 * d2p + g3 * d3m); break;
    case 3: pv = fc + (g1 * d1p + g2 * d2p - g3 * d3m); break;
    case 4: pv = fc - (g1 * d1m + g2 * d2m - g3 * d3p); break;
    case 5: pv = fc + (g1 * d1p - g2 * d2m + g3 * d3p); break;
    case 6: pv = fc - (g1 * d1m - g2 * d2p - g3 * d3p); break;
    default: pv = fc + (g1 * d1p + g2 * d2p + g3 * d3p); break;
  }
  return sgn(0) * pv;
}

// Plan entries [q0, q0 + n), one thread per (entry, variable).  INNER: the inner entries, into the scratch slots
// ([variable][nscr] doubles); otherwise the direct outer entries, into their
// ghost cells.
template <typename S, bool INNER>
__global__ void k_amr_fill_plan(const __grid_constant__ MeshDesc m, const GhostPlan *plan, int q0, int n, S *cc,
                                float *lo, S *prim, int ncc, double *scratch, int nscr) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const FillVar<S> fv(m, blockIdx.y, cc, lo, prim, ncc);
  const GhostPlan &g = plan[q0 + q];
  const Field f{fv.arr, fv.lo, sizeof(S) == 4};
  double *scr = scratch + (long long)blockIdx.y * nscr;
  const double val = plan_value(m, g, f, fv.fd, scr);
  if constexpr (INNER) scr[g.dst] = val;
  else store_value<S>(fv.arr, fv.lo, g.dst, val);
}

// Flux correction: a coarse block's boundary face whose neighbour across it
// is finer takes the area-weighted restriction of the 2^(d-1) fine face
// fluxes.  The faces and their fine faces are listed once per table upload
// (k_flux_plan, one thread per (block, direction, side, face)); the fix
// reads fine blocks' boundary faces and writes coarse blocks' boundary
// faces only.
struct FluxFix {
  long long dst;     // coarse face, offset in [nb][Pf]
  long long src[8];  // fine faces, slot off[2]*4 + off[1]*2 + off[0] (transverse offsets)
  double vv[8];      // their areas; 0 for unused slots
  int d;             // face direction
};

__device__ __forceinline__ bool flux_fix_entry(const MeshDesc &m, long long t, int F, FluxFix &fx) {
  if (t >= (long long)m.nb * 6 * F) return false;
  const int b = int(t / (6ll * F));
  const int rr = int(t - (long long)b * 6 * F);
  const int d = (rr / F) >> 1, s = (rr / F) & 1, a = rr % F;
  if (d >= m.ndim) return false;
  const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
  const int a1 = a % m.nx[t1], a2 = a / m.nx[t1];
  if (a2 >= m.nx[t2]) return false;
  const int L = m.blev[b];
  const int *bl = m.bloc + 3 * b;
  // the cell across the face, at level L
  int Gn[3];
  Gn[d] = bl[d] * m.nx[d] + (s ? m.nx[d] : -1);
  Gn[t1] = bl[t1] * m.nx[t1] + a1;
  Gn[t2] = bl[t2] * m.nx[t2] + a2;
  const int N = m.mesh_nx[d] << L;
  if ((Gn[d] < 0 || Gn[d] >= N) && m.bc[d][s] != BC_PERIODIC) return false;
  bool fl = false;
  Gn[d] = amr_map(Gn[d], N, m.bc[d][s], fl);
  int bxn[3];
  for (int q = 0; q < 3; q++) bxn[q] = Gn[q] / m.nx[q];
  if (table_at(m, L, bxn) != -1) return false;  // not finer across this face
  for (int q = 0; q < 8; q++) {
    fx.vv[q] = 0.0;
    fx.src[q] = 0;
  }
  for (int o2 = 0; o2 < 1 + (t2 < m.ndim); o2++)
    for (int o1 = 0; o1 < 1 + (t1 < m.ndim); o1++) {
      int Gf[3];
      const int Ff = 2 * (bl[d] * m.nx[d] + (s ? m.nx[d] : 0));
      Gf[d] = s ? Ff : Ff - 1;
      Gf[t1] = t1 < m.ndim ? 2 * (bl[t1] * m.nx[t1] + a1) + o1 : 0;
      Gf[t2] = t2 < m.ndim ? 2 * (bl[t2] * m.nx[t2] + a2) + o2 : 0;
      bool f2 = false;
      Gf[d] = amr_map(Gf[d], m.mesh_nx[d] << (L + 1), m.bc[d][s], f2);
      int bf[3], lf[3];
      for (int q = 0; q < 3; q++) bf[q] = Gf[q] / m.nx[q];
      const int e = table_at(m, L + 1, bf);
      if (e < 0) return false;  // not a leaf one level finer: the mesh is not 2:1 balanced
      for (int q = 0; q < 3; q++) lf[q] = Gf[q] - bf[q] * m.nx[q] + m.g[q];
      if (!s) lf[d] += 1;  // the fine cell's high face
      int off[3] = {0, 0, 0};
      off[t1] = o1;
      off[t2] = o2;
      const int slot = off[2] * 4 + off[1] * 2 + off[0];
      fx.vv[slot] = blk_area(m, e, d);
      fx.src[slot] = (long long)e * m.Pf + fidx(m, lf[2], lf[1], lf[0]);
    }
  int lc[3];
  lc[d] = m.g[d] + (s ? m.nx[d] : 0);
  lc[t1] = m.g[t1] + a1;
  lc[t2] = m.g[t2] + a2;
  fx.dst = (long long)b * m.Pf + fidx(m, lc[2], lc[1], lc[0]);
  fx.d = d;
  return true;
}

// Count (fixes null) or list the flux fixes of the current tables.
__global__ void k_flux_plan(const __grid_constant__ MeshDesc m, int F, FluxFix *fixes, int *count) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  FluxFix fx;
  if (!flux_fix_entry(m, t, F, fx)) return;
  const int q = atomicAdd(count, 1);
  if (fixes) fixes[q] = fx;
}

// One thread per (fix, conserved variable).
template <typename S>
__global__ void k_flux_correct(const __grid_constant__ MeshDesc m, const FluxFix *fixes, int n, S *flux, int ncc) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int v = blockIdx.y;
  const FluxFix &fx = fixes[q];
  const long long NF = (long long)m.nb * m.Pf;
  S *fv = flux + ((long long)fx.d * ncc + v) * NF;
  double tt[8], vv[8];
  for (int k = 0; k < 8; k++) vv[k] = fx.vv[k];
  for (int k = 0; k < 8; k++) tt[k] = vv[k] > 0.0 ? vv[k] * double(fv[fx.src[k]]) : 0.0;
  fv[fx.dst] = S(restrict8(tt, vv));
}

// AMRLoehner on one field of a container: one CTA per block, one thread per
// (k, j) row; the block's flag is the maximum of the row flags.  With
// several criteria the tag is the maximum over them (combine: max into tags).
__global__ void k_amr_tag(const __grid_constant__ MeshDesc m, Field f, double refine_tol, double derefine_tol,
                          double filter, int max_level, int combine, int *tags) {
  __shared__ int flag_sh;
  __shared__ unsigned long long max_sh;
  const int b = blockIdx.x;
  if (threadIdx.x == 0) max_sh = 0ull;
  __syncthreads();
  const int nd = m.ndim;
  const double dxq[3] = {blk_dx(m, b, 0), blk_dx(m, b, 1), blk_dx(m, b, 2)};
  const long long base = (long long)b * m.P;
  const long long st[3] = {1, m.np[0], (long long)m.np[0] * m.np[1]};
  auto U = [&](long long n) { return fetch(f, base + n); };
  // central first derivative along p at cell n
  auto Dv = [&](int p, long long n) { return 0.5 * (U(n + st[p]) - U(n - st[p])) / dxq[p]; };
  // One thread per cell.  The reference flags each row by its largest error
  // and the block by the largest row flag; the flag grows with the error, so
  // that is the flag of the block's largest error, taken here as the maximum
  // of the squared ratios (non-negative doubles order as their bit patterns).
  const int ncell = m.nx[0] * m.nx[1] * m.nx[2];
  double max_err_2 = 0.;
  for (int c = threadIdx.x; c < ncell; c += blockDim.x) {
    const int i = m.g[0] + c % m.nx[0], j = m.g[1] + (c / m.nx[0]) % m.nx[1], k = m.g[2] + c / (m.nx[0] * m.nx[1]);
    const long long n = cidx(m, k, j, i);
    double numerator = 0.0, denominator = 1.e-12;
    for (int q = 0; q < nd; q++) {
      const long long sq = st[q];
      for (int p = 0; p < nd; p++) {
        const long long sp = st[p];
        const double dpp = Dv(p, n + sq), dpm = Dv(p, n - sq);
        const double num = 0.5 * (dpp - dpm) / dxq[q];
        numerator += num * num;
        const double denom =
            0.5 * (fabs(dpp) + fabs(dpm)) / dxq[p] +
            filter * (fabs(U(n + sq)) + fabs(U(n - sq)) + fabs(U(n - sp)) + fabs(U(n + sp))) / (dxq[q] * dxq[p]);
        denominator += denom * denom;
      }
    }
    if (denominator != 0.0) {
      const double ratio = numerator / denominator;
      max_err_2 = (max_err_2 < ratio) ? ratio : max_err_2;
    }
  }
  atomicMax(&max_sh, (unsigned long long)__double_as_longlong(max_err_2));
  __syncthreads();
  if (threadIdx.x == 0) {
    const double max_err = sqrt(__longlong_as_double((long long)max_sh));
    int flag = 0;
    if (max_err > refine_tol && m.blev[b] < max_level) flag = 1;
    if (max_err < derefine_tol) flag = -1;
    flag_sh = flag;
  }
  if (threadIdx.x == 0) tags[b] = combine ? max(tags[b], flag_sh) : flag_sh;
}

// Remap after a remesh: every interior cell of the new leaves takes the level
// value of the old mesh (copy, prolongation or restriction).
template <typename S>
__global__ void __launch_bounds__(kThreads, kLvBlocks) k_amr_remap(const __grid_constant__ MeshDesc mo, const S *occ, const float *olo, const S *oprim,
                            int nnew, const int *nlev, const int *nloc, S *ncc_out, float *nlo, S *nprim, int ncc,
                            int *err) {
  // one thread per (new interior cell, variable): blockIdx.y runs over the
  // ncc conserved variables, then the NPRIM primitives
  const unsigned cells = unsigned(mo.nx[0]) * unsigned(mo.nx[1]) * unsigned(mo.nx[2]);
  const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cells * unsigned(nnew)) return;
  const int v = blockIdx.y;
  const int q = int(t / cells);
  unsigned r = t - unsigned(q) * cells;
  const int i = mo.g[0] + int(r % unsigned(mo.nx[0]));
  r /= unsigned(mo.nx[0]);
  const int j = mo.g[1] + int(r % unsigned(mo.nx[1]));
  const int k = mo.g[2] + int(r / unsigned(mo.nx[1]));
  const int G0 = nloc[3 * q] * mo.nx[0] + (i - mo.g[0]);
  const int G1 = nloc[3 * q + 1] * mo.nx[1] + (j - mo.g[1]);
  const int G2 = nloc[3 * q + 2] * mo.nx[2] + (k - mo.g[2]);
  const int L = nlev[q];
  constexpr bool F32 = sizeof(S) == 4;
  const long long NPo = (long long)mo.nb * mo.P, NPn = (long long)nnew * mo.P;
  const long long dst = (long long)q * mo.P + cidx(mo, k, j, i);
  if (v < ncc) {
    const Field f{occ + v * NPo, (F32 && v == CENER) ? olo : nullptr, F32};
    const int fd = (v >= CMOM0 && v <= CMOM2) ? v - CMOM0 : (v >= CMAGC0 ? v - CMAGC0 : -1);
    const double val = level_value_at<kMaxDepth>(mo, L, G0, G1, G2, f, fd, err);
    store_value<S>(ncc_out + v * NPn, v == CENER ? nlo : nullptr, dst, val);
  } else {
    const int pv = v - ncc;
    const Field f{oprim + pv * NPo, nullptr, F32};
    const double val = level_value_at<kMaxDepth>(mo, L, G0, G1, G2, f, pv <= PVEL2 ? pv : -1, err);
    store_value<S>(nprim + pv * NPn, nullptr, dst, val);
  }
}

// Ghost faces of component e (active components only): the face value of
// the position they cover.  The block's own faces, boundary faces included,
// are left alone; the kernel reads only faces that leaves own.
template <typename S>
__global__ void k_amr_fill_ghost_faces(const __grid_constant__ MeshDesc m, S *fc, int e, int *err) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)m.nb * m.Pf) return;
  const int b = int(t / m.Pf);
  long long r = t - (long long)b * m.Pf;
  const int i = int(r % m.nf[0]);
  r /= m.nf[0];
  const int j = int(r % m.nf[1]);
  const int k = int(r / m.nf[1]);
  const int loc[3] = {i, j, k};
  for (int d = 0; d < 3; d++)
    if (loc[d] >= m.np[d] + (d == e ? 1 : 0)) return;  // outside this component's extent
  bool interior = true;
  for (int d = 0; d < 3; d++) {
    const int hi = m.g[d] + m.nx[d] - 1 + (d == e ? 1 : 0);
    if (loc[d] < m.g[d] || loc[d] > hi) interior = false;
  }
  if (interior) return;
  int G[3];
  for (int d = 0; d < 3; d++) G[d] = m.bloc[3 * b + d] * m.nx[d] + (loc[d] - m.g[d]);
  const FaceField f{fc, (long long)m.nb * m.Pf, sizeof(S) == 4};
  int calls = 0;
  const double v = face_value<kMaxDepth>(m, e, m.blev[b], G[0], G[1], G[2], f, err, &calls);
  fc[e * f.NF + (long long)b * m.Pf + fidx(m, k, j, i)] = S(v);
}

// Edge-EMF correction at fine/coarse boundaries (the face-field part of the
// flux correction, kamayan_driver.cpp:198-207).  An edge on a block's boundary
// where any of the cells around it (four in 3D, the four quadrants of a
// corner in 2D) is covered by finer leaves takes the length-weighted
// restriction of the collinear fine EMFs, read from the fine leaf holding the
// first such cell (order (-,-), (+,-), (-,+), (+,+) over the edge's two
// transverse axes).  Every block holding the edge computes the same value, so
// same-level neighbours keep identical copies of their shared faces.  Reads
// the EMFs as computed (eo), writes the corrected ones (emf).
template <typename S>
__global__ void k_emf_correct(const __grid_constant__ MeshDesc m, const S *eo, S *emf, int E) {
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (tid >= (long long)m.nb * 3 * E) return;
  const int b = int(tid / (3ll * E));
  const int rr = int(tid - (long long)b * 3 * E);
  const int t = rr / E, idx = rr % E;
  if (m.ndim == 2 && t != 2) return;  // 2D has z-edges only
  const int p = (t + 1) % 3, q = (t + 2) % 3;
  const int np_ = m.nx[p] + 1, nq_ = m.nx[q] + 1;
  const int ap = idx % np_, aq = (idx / np_) % nq_, at = idx / (np_ * nq_);
  if (at >= m.nx[t]) return;
  if (ap != 0 && ap != m.nx[p] && aq != 0 && aq != m.nx[q]) return;  // not on the block boundary
  const int L = m.blev[b];
  const int *bl = m.bloc + 3 * b;
  const int Ep = bl[p] * m.nx[p] + ap, Eq = bl[q] * m.nx[q] + aq, Et = bl[t] * m.nx[t] + at;
  const long long NF = (long long)m.nb * m.Pf;
  for (int s = 0; s < 4; s++) {
    const int dp = s & 1, dq = s >> 1;
    int Gc[3];
    Gc[p] = Ep - 1 + dp;
    Gc[q] = Eq - 1 + dq;
    Gc[t] = Et;
    bool skip = false;
    for (int w = 0; w < 2; w++) {
      const int d = w ? q : p;
      const int N = m.mesh_nx[d] << L;
      if (Gc[d] < 0 || Gc[d] >= N) {
        if (m.bc[d][Gc[d] < 0 ? 0 : 1] != BC_PERIODIC) skip = true;
        else Gc[d] = ((Gc[d] % N) + N) % N;
      }
    }
    if (skip) continue;
    int bxc[3];
    for (int d = 0; d < 3; d++) bxc[d] = Gc[d] / m.nx[d];
    if (table_at(m, L, bxc) != -1) continue;
    int Fc[3];
    Fc[p] = 2 * Gc[p] + (dp ? 0 : 1);
    Fc[q] = 2 * Gc[q] + (dq ? 0 : 1);
    Fc[t] = t < m.ndim ? 2 * Et : 0;
    double tt[8] = {0, 0, 0, 0, 0, 0, 0, 0}, vv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool ok = true;
    for (int o = 0; o < 1 + (t < m.ndim); o++) {
      int Ff[3] = {Fc[0], Fc[1], Fc[2]};
      Ff[t] += o;
      int bf[3];
      for (int d = 0; d < 3; d++) bf[d] = Ff[d] / m.nx[d];
      const int fe = table_at(m, L + 1, bf);
      if (fe < 0) {
        ok = false;
        break;
      }
      int lf[3];
      for (int d = 0; d < 3; d++) lf[d] = Ff[d] - bf[d] * m.nx[d] + m.g[d];
      if (!dp) lf[p] += 1;
      if (!dq) lf[q] += 1;
      const int slot = t == 0 ? o : t == 1 ? 2 * o : 4 * o;
      const double len = blk_dx(m, fe, t);
      vv[slot] = len;
      tt[slot] = len * double(eo[t * NF + (long long)fe * m.Pf + fidx(m, lf[2], lf[1], lf[0])]);
    }
    if (!ok) continue;
    int le[3];
    le[p] = m.g[p] + ap;
    le[q] = m.g[q] + aq;
    le[t] = m.g[t] + at;
    emf[t * NF + (long long)b * m.Pf + fidx(m, le[2], le[1], le[0])] = S(restrict8(tt, vv));
    return;
  }
}

// Faces of the new leaves after a remesh, every component, boundary faces
// included: the face value of the old mesh.
template <typename S>
__global__ void k_amr_remap_faces(const __grid_constant__ MeshDesc mo, const S *ofc, int nnew, const int *nlev,
                                  const int *nloc, S *nfc, int *err) {
  const long long per = (long long)(mo.nx[0] + 1) * (mo.nx[1] + 1) * (mo.nx[2] + 1);
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= per * 3 * nnew) return;
  const int q = int(t / (per * 3));
  long long r = t - (long long)q * per * 3;
  const int e = int(r / per);
  r -= (long long)e * per;
  const int i = int(r % (mo.nx[0] + 1));
  r /= (mo.nx[0] + 1);
  const int j = int(r % (mo.nx[1] + 1));
  const int k = int(r / (mo.nx[1] + 1));
  // own faces: nx + 1 along e when e is active, nx across
  const int ext[3] = {mo.nx[0] + (e == 0 ? 1 : 0), mo.nx[1] + (e == 1 && mo.ndim > 1 ? 1 : 0),
                      mo.nx[2] + (e == 2 && mo.ndim > 2 ? 1 : 0)};
  if (i >= ext[0] || j >= ext[1] || k >= ext[2]) return;
  const int G0 = nloc[3 * q] * mo.nx[0] + i, G1 = nloc[3 * q + 1] * mo.nx[1] + j, G2 = nloc[3 * q + 2] * mo.nx[2] + k;
  const FaceField f{ofc, (long long)mo.nb * mo.Pf, sizeof(S) == 4};
  int calls = 0;
  const double v = face_value<kMaxDepth>(mo, e, nlev[q], G0, G1, G2, f, err, &calls);
  nfc[e * (long long)nnew * mo.Pf + (long long)q * mo.Pf + fidx(mo, k + mo.g[2], j + mo.g[1], i + mo.g[0])] = S(v);
}

// Morton key of a leaf's lower corner at the finest level, level in the low bits.
uint64_t morton_key(int x0, int y0, int z0, int level, int maxl) {
  const int sh = maxl - level;
  const uint64_t x = uint64_t(x0) << sh, y = uint64_t(y0) << sh, z = uint64_t(z0) << sh;
  uint64_t key = 0;
  for (int bit = 0; bit < 20; bit++) {
    key |= ((x >> bit) & 1ull) << (3 * bit);
    key |= ((y >> bit) & 1ull) << (3 * bit + 1);
    key |= ((z >> bit) & 1ull) << (3 * bit + 2);
  }
  return (key << 5) | uint64_t(level);
}

}  // namespace

// Level tables and leaf arrays to the device; MeshDesc points at them.
int amr_upload(kmy_ctx *c) {
  c->amr.gen++;
  AmrHost &a = c->amr;
  MeshDesc &m = c->m;
  const int nb = int(a.lev.size());
  const int nlev = a.max_level + 1;
  std::vector<int> tabs;
  long long total = 0;
  for (int L = 0; L < nlev; L++) {
    m.tab_off[L] = int(total);
    long long n = 1;
    for (int d = 0; d < 3; d++) {
      m.tab_dim[L][d] = d < m.ndim ? (m.nbx[d] << L) : 1;
      n *= m.tab_dim[L][d];
    }
    total += n;
    if (total > kMaxTable) {
      c->err = "adaptive mesh: level tables exceed " + std::to_string(kMaxTable) + " entries";
      return KMY_ERR_BAD_PARAM;
    }
  }
  tabs.assign(size_t(total), -2);
  for (int b = 0; b < nb; b++) {
    const int Lb = a.lev[b];
    for (int L = 0; L <= Lb; L++) {
      int q[3];
      for (int d = 0; d < 3; d++) q[d] = d < m.ndim ? (a.loc[3 * b + d] >> (Lb - L)) : 0;
      const long long idx = m.tab_off[L] + ((long long)q[2] * m.tab_dim[L][1] + q[1]) * m.tab_dim[L][0] + q[0];
      tabs[size_t(idx)] = L == Lb ? b : -1;
    }
  }
  dfree(c, a.d_blev);
  dfree(c, a.d_bloc);
  dfree(c, a.d_tabs);
  dfree(c, a.d_tags);
  a.d_blev = a.d_bloc = a.d_tabs = a.d_tags = nullptr;
  int rc = dalloc(c, reinterpret_cast<void **>(&a.d_blev), sizeof(int) * nb);
  if (!rc) rc = dalloc(c, reinterpret_cast<void **>(&a.d_bloc), sizeof(int) * 3 * nb);
  if (!rc) rc = dalloc(c, reinterpret_cast<void **>(&a.d_tabs), sizeof(int) * size_t(total));
  if (!rc) rc = dalloc(c, reinterpret_cast<void **>(&a.d_tags), sizeof(int) * nb);
  if (rc) return rc;
  rc = cuda_check(c, cudaMemcpyAsync(a.d_blev, a.lev.data(), sizeof(int) * nb, cudaMemcpyHostToDevice, c->stream),
                  "amr levels");
  if (!rc)
    rc = cuda_check(c, cudaMemcpyAsync(a.d_bloc, a.loc.data(), sizeof(int) * 3 * nb, cudaMemcpyHostToDevice,
                                       c->stream), "amr locations");
  if (!rc)
    rc = cuda_check(c, cudaMemcpyAsync(a.d_tabs, tabs.data(), sizeof(int) * size_t(total), cudaMemcpyHostToDevice,
                                       c->stream), "amr tables");
  // pageable sources: wait so the host vectors may go
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "amr upload");
  if (rc) return rc;
  m.nb = nb;
  m.blev = a.d_blev;
  m.bloc = a.d_bloc;
  m.tabs = a.d_tabs;
  m.nlev = nlev;
  // the ghost plan of the new tables: count, allocate, fill
  dfree(c, a.d_plan);
  dfree(c, a.d_plan_scr);
  dfree(c, a.d_copy);
  a.d_plan = nullptr;
  a.d_plan_scr = nullptr;
  a.d_copy = nullptr;
  a.plan_n = a.plan_deep = a.plan_inner = a.copy_n = 0;
  const long long cells = (long long)m.nb * m.P;
  if (cells >= (1LL << 32)) {
    c->err = "adaptive mesh: more than 2^32 padded cells";
    return KMY_ERR_BAD_PARAM;
  }
  if (!a.d_plan_n) rc = dalloc(c, reinterpret_cast<void **>(&a.d_plan_n), 4 * sizeof(int));
  int count[4] = {0, 0, 0, 0};
  if (!rc) rc = cuda_check(c, cudaMemsetAsync(a.d_plan_n, 0, 4 * sizeof(int), c->stream), "plan count");
  if (!rc) {
    k_amr_plan<<<nblk(cells), kThreads, 0, c->stream>>>(m, nullptr, nullptr, a.d_plan_n, 0, 0);
    c->launches++;
    rc = cuda_check(c, cudaMemcpyAsync(count, a.d_plan_n, 4 * sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                    "plan count");
  }
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "plan count");
  if (rc) return rc;
  const long long nplan = (long long)count[0] + count[1] + count[2];
  if (nplan > 0) rc = dalloc(c, &a.d_plan, sizeof(GhostPlan) * size_t(nplan));
  if (!rc && count[2] > 0)
    rc = dalloc(c, reinterpret_cast<void **>(&a.d_plan_scr), sizeof(double) * size_t(c->ncc + NPRIM) * count[2]);
  if (!rc && count[3] > 0) rc = dalloc(c, &a.d_copy, sizeof(GhostCopy) * size_t(count[3]));
  if (!rc) rc = cuda_check(c, cudaMemsetAsync(a.d_plan_n, 0, 4 * sizeof(int), c->stream), "plan fill");
  if (!rc && (nplan > 0 || count[3] > 0)) {
    k_amr_plan<<<nblk(cells), kThreads, 0, c->stream>>>(m, static_cast<GhostPlan *>(a.d_plan),
                                                        static_cast<GhostCopy *>(a.d_copy), a.d_plan_n, count[0],
                                                        count[1]);
    c->launches++;
    rc = cuda_check(c, cudaGetLastError(), "plan fill");
  }
  if (!rc) {
    a.plan_n = count[0];
    a.plan_deep = count[1];
    a.plan_inner = count[2];
    a.copy_n = count[3];
  }
  // the flux fixes of the new tables: count, allocate, fill
  dfree(c, a.d_fix);
  a.d_fix = nullptr;
  a.fix_n = 0;
  int F = 1;
  for (int d = 0; d < m.ndim; d++) F = std::max(F, m.nx[(d + 1) % 3] * m.nx[(d + 2) % 3]);
  const long long nfix = (long long)m.nb * 6 * F;
  int nf = 0;
  if (!rc) rc = cuda_check(c, cudaMemsetAsync(a.d_plan_n, 0, sizeof(int), c->stream), "flux plan count");
  if (!rc) {
    k_flux_plan<<<nblk(nfix), kThreads, 0, c->stream>>>(m, F, nullptr, a.d_plan_n);
    c->launches++;
    rc = cuda_check(c, cudaMemcpyAsync(&nf, a.d_plan_n, sizeof(int), cudaMemcpyDeviceToHost, c->stream),
                    "flux plan count");
  }
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "flux plan count");
  if (!rc && nf > 0) {
    rc = dalloc(c, &a.d_fix, sizeof(FluxFix) * size_t(nf));
    if (!rc) rc = cuda_check(c, cudaMemsetAsync(a.d_plan_n, 0, sizeof(int), c->stream), "flux plan");
    if (!rc) {
      k_flux_plan<<<nblk(nfix), kThreads, 0, c->stream>>>(m, F, static_cast<FluxFix *>(a.d_fix), a.d_plan_n);
      c->launches++;
      rc = cuda_check(c, cudaGetLastError(), "flux plan");
    }
    if (!rc) a.fix_n = nf;
  }
  return rc;
}

// Initial leaves: every block of the root grid at level 0, lexicographic.
int amr_setup(kmy_ctx *c) {
  AmrHost &a = c->amr;
  const MeshDesc &m = c->m;
  a.lev.assign(m.nb, 0);
  a.loc.assign(size_t(3) * m.nb, 0);
  a.cnt.assign(m.nb, 0);
  for (int b = 0; b < m.nb; b++) {
    a.loc[3 * b] = b % m.nbx[0];
    a.loc[3 * b + 1] = (b / m.nbx[0]) % m.nbx[1];
    a.loc[3 * b + 2] = b / (m.nbx[0] * m.nbx[1]);
  }
  int rc = dalloc(c, reinterpret_cast<void **>(&a.d_err), sizeof(int));
  if (!rc) rc = amr_upload(c);
  return rc;
}

int launch_amr_fill_ghosts(kmy_ctx *c, Container &ct) {
  const MeshDesc &m = c->m;
  const unsigned nvar = unsigned(c->ncc + NPRIM);
  const int ncp = c->amr.copy_n;
  if (ncp > 0) {
    const dim3 grid(nblk(ncp), nvar);
    const GhostCopy *cp = static_cast<const GhostCopy *>(c->amr.d_copy);
    if (c->esz == 8)
      k_amr_fill_copy<double><<<grid, kThreads, 0, c->stream>>>(m, cp, ncp, (double *)ct.cc, nullptr,
                                                                (double *)c->prim, c->ncc);
    else
      k_amr_fill_copy<float><<<grid, kThreads, 0, c->stream>>>(m, cp, ncp, (float *)ct.cc, (float *)ct.ener_lo,
                                                               (float *)c->prim, c->ncc);
    c->launches++;
  }
  const GhostPlan *plan = static_cast<const GhostPlan *>(c->amr.d_plan);
  const int n0 = c->amr.plan_n, n1 = c->amr.plan_deep, n2 = c->amr.plan_inner;
  double *scr = c->amr.d_plan_scr;
  // inner entries first: the direct ones read their scratch slots
  if (n2 > 0) {
    const dim3 pgrid(nblk(n2), nvar);
    if (c->esz == 8)
      k_amr_fill_plan<double, true><<<pgrid, kThreads, 0, c->stream>>>(m, plan, n0 + n1, n2, (double *)ct.cc,
                                                                       nullptr, (double *)c->prim, c->ncc, scr, n2);
    else
      k_amr_fill_plan<float, true><<<pgrid, kThreads, 0, c->stream>>>(m, plan, n0 + n1, n2, (float *)ct.cc,
                                                                      (float *)ct.ener_lo, (float *)c->prim, c->ncc,
                                                                      scr, n2);
    c->launches++;
  }
  if (n0 > 0) {
    const dim3 pgrid(nblk(n0), nvar);
    if (c->esz == 8)
      k_amr_fill_plan<double, false><<<pgrid, kThreads, 0, c->stream>>>(m, plan, 0, n0, (double *)ct.cc, nullptr,
                                                                        (double *)c->prim, c->ncc, scr, n2);
    else
      k_amr_fill_plan<float, false><<<pgrid, kThreads, 0, c->stream>>>(m, plan, 0, n0, (float *)ct.cc,
                                                                       (float *)ct.ener_lo, (float *)c->prim,
                                                                       c->ncc, scr, n2);
    c->launches++;
  }
  if (n1 > 0) {
    const dim3 pgrid(nblk(n1), nvar);
    if (c->esz == 8)
      k_amr_fill_plan_deep<double><<<pgrid, kThreads, 0, c->stream>>>(m, plan, n0, n1, (double *)ct.cc, nullptr,
                                                                      (double *)c->prim, c->ncc, c->amr.d_err);
    else
      k_amr_fill_plan_deep<float><<<pgrid, kThreads, 0, c->stream>>>(m, plan, n0, n1, (float *)ct.cc,
                                                                     (float *)ct.ener_lo, (float *)c->prim, c->ncc,
                                                                     c->amr.d_err);
    c->launches++;
  }
  if (c->prm.mhd) {
    const long long nf = (long long)m.nb * m.Pf;
    for (int e = 0; e < m.ndim; e++) {
      if (c->esz == 8)
        k_amr_fill_ghost_faces<double><<<nblk(nf), kThreads, 0, c->stream>>>(m, (double *)ct.fc, e, c->amr.d_err);
      else
        k_amr_fill_ghost_faces<float><<<nblk(nf), kThreads, 0, c->stream>>>(m, (float *)ct.fc, e, c->amr.d_err);
      c->launches++;
    }
  }
  return cuda_check(c, cudaGetLastError(), "amr fill_ghosts");
}

int launch_emf_correct(kmy_ctx *c, Container &md0) {
  const MeshDesc &m = c->m;
  AmrHost &a = c->amr;
  if (!c->prm.mhd || m.ndim < 2 || !md0.emf) return KMY_OK;
  const size_t bytes = c->esz * 3 * size_t(m.nb) * m.Pf;
  if (a.emf_tmp_bytes != bytes) {
    dfree(c, a.d_emf_tmp);
    a.d_emf_tmp = nullptr;
    a.emf_tmp_bytes = 0;
    const int rc = dalloc(c, &a.d_emf_tmp, bytes);
    if (rc) return rc;
    a.emf_tmp_bytes = bytes;
  }
  int rc = cuda_check(c, cudaMemcpyAsync(a.d_emf_tmp, md0.emf, bytes, cudaMemcpyDeviceToDevice, c->stream),
                      "emf copy");
  if (rc) return rc;
  int E = 1;
  for (int t = 0; t < 3; t++) E = std::max(E, (m.nx[(t + 1) % 3] + 1) * (m.nx[(t + 2) % 3] + 1) * m.nx[t]);
  const long long n = (long long)m.nb * 3 * E;
  if (c->esz == 8)
    k_emf_correct<double><<<nblk(n), kThreads, 0, c->stream>>>(m, (const double *)a.d_emf_tmp, (double *)md0.emf, E);
  else
    k_emf_correct<float><<<nblk(n), kThreads, 0, c->stream>>>(m, (const float *)a.d_emf_tmp, (float *)md0.emf, E);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "emf_correct");
}


int launch_flux_correct(kmy_ctx *c) {
  const MeshDesc &m = c->m;
  const int n = c->amr.fix_n;
  if (!c->flux || n == 0) return KMY_OK;
  const dim3 grid(nblk(n), unsigned(c->ncc));
  const FluxFix *fx = static_cast<const FluxFix *>(c->amr.d_fix);
  if (c->esz == 8)
    k_flux_correct<double><<<grid, kThreads, 0, c->stream>>>(m, fx, n, (double *)c->flux, c->ncc);
  else
    k_flux_correct<float><<<grid, kThreads, 0, c->stream>>>(m, fx, n, (float *)c->flux, c->ncc);
  c->launches++;
  return cuda_check(c, cudaGetLastError(), "flux_correct");
}

int launch_amr_tag(kmy_ctx *c, Container &ct) {
  const MeshDesc &m = c->m;
  const AmrHost &a = c->amr;
  const long long NP = (long long)m.nb * m.P;
  for (size_t i = 0; i < a.crits.size(); i++) {
    const AmrCriterion &cr = a.crits[i];
    Field f{nullptr, nullptr, c->esz == 4};
    if (cr.field == "pres") {
      f.p = static_cast<const char *>(c->prim) + c->esz * NP * PPRES;
    } else if (cr.field == "ener") {
      f.p = static_cast<const char *>(ct.cc) + c->esz * NP * CENER;
      f.lo = static_cast<const float *>(ct.ener_lo);
    } else {
      f.p = static_cast<const char *>(ct.cc) + c->esz * NP * CDENS;
    }
    k_amr_tag<<<m.nb, kThreads, 0, c->stream>>>(m, f, cr.refine_tol, cr.derefine_tol, cr.filter, cr.max_level,
                                                 i > 0, a.d_tags);
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "amr tag");
}

// Parthenon's tree update, restated: refine the leaves tagged for refinement
// below max_level, restore 2:1 balance across faces, edges and corners by
// refining coarser neighbours, then (allow_derefine) merge sibling groups
// whose members were tagged for derefinement derefine_count times in a row
// when the merged parent keeps the balance.  New leaves are ordered by the
// Morton key of their lower corner and get their data from the old mesh.
int amr_remesh(kmy_ctx *c, bool allow_derefine, bool *changed_out, DevClock *clock_out) {
  AmrHost &a = c->amr;
  MeshDesc &m = c->m;
  const int nd = m.ndim;
  const int nb = m.nb;
  *changed_out = false;
  // pinned staging: [the clock] [error flag] [tags]
  const size_t cb = clock_out ? sizeof(DevClock) : 0;
  char *stage = static_cast<char *>(host_pin(c, cb + sizeof(int) * (size_t(nb) + 1)));
  if (!stage) return KMY_ERR_OOM;
  int *pin = reinterpret_cast<int *>(stage + cb);
  int rc = cuda_check(c, cudaMemcpyAsync(pin + 1, a.d_tags, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->stream),
                      "amr tags");
  if (!rc) rc = cuda_check(c, cudaMemcpyAsync(pin, a.d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream), "amr err");
  if (!rc && clock_out)
    rc = cuda_check(c, cudaMemcpyAsync(stage, c->clock, sizeof(DevClock), cudaMemcpyDeviceToHost, c->stream),
                    "amr clock");
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "amr tags sync");
  if (rc) return rc;
  if (clock_out) std::memcpy(clock_out, stage, sizeof(DevClock));
  const std::vector<int> tags(pin + 1, pin + 1 + nb);
  bool any = false;
  rc = amr_count_tags(c, tags, pin[0], &any);
  if (rc || !any) return rc;
  return amr_remesh_apply(c, allow_derefine, tags, changed_out);
}

int amr_count_tags(kmy_ctx *c, const std::vector<int> &tags, int err, bool *any_out) {
  AmrHost &a = c->amr;
  *any_out = false;
  if (err) {
    c->err = "adaptive mesh: a level-value evaluation exceeded its depth or call budget (mesh not 2:1 balanced)";
    return KMY_ERR_STATE;
  }
  // derefinement counts; a step with no split candidate, a balanced tree and
  // no leaf due for derefinement leaves the mesh as it is
  bool any = !a.balanced;
  for (int b = 0; b < c->m.nb; b++) {
    a.cnt[b] = tags[b] == -1 ? a.cnt[b] + 1 : 0;
    if ((tags[b] == 1 && a.lev[b] < a.max_level) || (a.lev[b] > 0 && a.cnt[b] >= a.derefine_count)) any = true;
  }
  *any_out = any;
  return KMY_OK;
}

int amr_remesh_apply(kmy_ctx *c, bool allow_derefine, const std::vector<int> &tags, bool *changed_out,
                     const std::function<int()> &before_change) {
  AmrHost &a = c->amr;
  MeshDesc &m = c->m;
  const int nd = m.ndim;
  const int nb = m.nb;
  *changed_out = false;
  int rc = KMY_OK;
  typedef std::array<int, 4> Key;  // level, location
  std::map<Key, int> leaf;         // -> old leaf id, -1 for a new leaf
  for (int b = 0; b < nb; b++) leaf[{a.lev[b], a.loc[3 * b], a.loc[3 * b + 1], a.loc[3 * b + 2]}] = b;
  bool changed = false;
  auto child = [&](const Key &p, int o) {
    return Key{p[0] + 1, 2 * p[1] + (o & 1), nd > 1 ? 2 * p[2] + ((o >> 1) & 1) : 0,
               nd > 2 ? 2 * p[3] + ((o >> 2) & 1) : 0};
  };
  auto split = [&](const Key &k) {
    leaf.erase(k);
    for (int o = 0; o < (1 << nd); o++) leaf[child(k, o)] = -1;
    changed = true;
  };
  // the leaf covering block position p of level L, if it is at level <= L
  auto covering = [&](int L, int p0, int p1, int p2, Key &out) -> bool {
    int p[3] = {p0, p1, p2};
    for (int d = 0; d < nd; d++) {
      const int NB = m.nbx[d] << L;
      if (p[d] < 0 || p[d] >= NB) {
        if (m.bc[d][p[d] < 0 ? 0 : 1] != BC_PERIODIC) return false;
        p[d] = ((p[d] % NB) + NB) % NB;
      }
    }
    for (int l = L; l >= 0; l--) {
      const Key k = {l, p[0] >> (L - l), nd > 1 ? p[1] >> (L - l) : 0, nd > 2 ? p[2] >> (L - l) : 0};
      if (leaf.count(k)) {
        out = k;
        return true;
      }
    }
    return false;
  };
  for (int b = 0; b < nb; b++)
    if (tags[b] == 1 && a.lev[b] < a.max_level) split({a.lev[b], a.loc[3 * b], a.loc[3 * b + 1], a.loc[3 * b + 2]});
  // 2:1 balance.  Only splits can unbalance a balanced tree (derefinement
  // below checks its neighbours), so a step without splits skips the pass.
  for (bool again = changed || !a.balanced; again;) {
    again = false;
    std::vector<Key> keys;
    for (auto &kv : leaf) keys.push_back(kv.first);
    for (const Key &k : keys) {
      if (!leaf.count(k)) continue;
      for (int dz = -(nd > 2); dz <= (nd > 2); dz++)
        for (int dy = -(nd > 1); dy <= (nd > 1); dy++)
          for (int dxo = -1; dxo <= 1; dxo++) {
            if (!dxo && !dy && !dz) continue;
            Key n;
            if (!covering(k[0], k[1] + dxo, k[2] + dy, k[3] + dz, n)) continue;
            if (n[0] < k[0] - 1) {
              split(n);
              again = true;
            }
          }
    }
  }
  a.balanced = true;
  if (allow_derefine) {
    std::map<Key, int> parents;
    for (auto &kv : leaf) {
      const Key &k = kv.first;
      if (k[0] == 0 || kv.second < 0) continue;
      if (a.cnt[kv.second] < a.derefine_count) continue;
      parents[{k[0] - 1, k[1] >> 1, k[2] >> 1, k[3] >> 1}]++;
    }
    for (auto &pk : parents) {
      if (pk.second != (1 << nd)) continue;
      const Key &p = pk.first;
      bool ok = true;
      for (int dz = -(nd > 2); dz <= (nd > 2) && ok; dz++)
        for (int dy = -(nd > 1); dy <= (nd > 1) && ok; dy++)
          for (int dxo = -1; dxo <= 1 && ok; dxo++) {
            if (!dxo && !dy && !dz) continue;
            Key n;
            if (covering(p[0], p[1] + dxo, p[2] + dy, p[3] + dz, n)) continue;
            // finer there: each child one level below p must be a leaf
            int q[3] = {p[1] + dxo, p[2] + dy, p[3] + dz};
            for (int d = 0; d < nd; d++) {
              const int NB = m.nbx[d] << p[0];
              if (q[d] < 0 || q[d] >= NB) q[d] = ((q[d] % NB) + NB) % NB;
            }
            const Key qp = {p[0], q[0], q[1], q[2]};
            for (int o = 0; o < (1 << nd) && ok; o++)
              if (!leaf.count(child(qp, o))) ok = false;
          }
      if (!ok) continue;
      for (int o = 0; o < (1 << nd); o++) leaf.erase(child(p, o));
      leaf[p] = -1;
      changed = true;
    }
  }
  if (!changed) return KMY_OK;
  // the new tree differs: the caller's last word before the device state is
  // remapped
  if (before_change) {
    if (const int r = before_change()) return r;
  }

  std::vector<std::pair<uint64_t, Key>> order;
  int maxl = 0;
  for (auto &kv : leaf) maxl = std::max(maxl, kv.first[0]);
  for (auto &kv : leaf) order.push_back({morton_key(kv.first[1], kv.first[2], kv.first[3], kv.first[0], maxl), kv.first});
  std::sort(order.begin(), order.end());
  const int nnew = int(order.size());
  std::vector<int> nlev(nnew), nloc(size_t(3) * nnew), ncnt(nnew, 0);
  for (int q = 0; q < nnew; q++) {
    const Key &k = order[q].second;
    nlev[q] = k[0];
    for (int d = 0; d < 3; d++) nloc[3 * q + d] = k[1 + d];
    const int old = leaf.find(k)->second;
    if (old >= 0) ncnt[q] = a.cnt[old];
  }

  // remap base and the primitives through the old mesh's level values
  const MeshDesc mo = m;
  const size_t n_new = size_t(nnew) * m.P;
  int *d_nlev = nullptr, *d_nloc = nullptr;
  Container nb_ct;
  void *nprim = nullptr;
  rc = dalloc(c, reinterpret_cast<void **>(&d_nlev), sizeof(int) * nnew);
  if (!rc) rc = dalloc(c, reinterpret_cast<void **>(&d_nloc), sizeof(int) * 3 * nnew);
  if (!rc) rc = dalloc(c, &nb_ct.cc, c->esz * c->ncc * n_new);
  if (!rc && c->esz == 4) rc = dalloc(c, &nb_ct.ener_lo, 4 * n_new);
  if (!rc) rc = dalloc(c, &nprim, c->esz * NPRIM * n_new);
  const size_t nf_new = size_t(nnew) * m.Pf;
  if (!rc && c->prm.mhd) rc = dalloc(c, &nb_ct.fc, c->esz * 3 * nf_new);
  if (!rc && c->prm.mhd) rc = dalloc(c, &nb_ct.emf, c->esz * 3 * nf_new);
  if (!rc)
    rc = cuda_check(c, cudaMemcpyAsync(d_nlev, nlev.data(), sizeof(int) * nnew, cudaMemcpyHostToDevice, c->stream),
                    "remap levels");
  if (!rc)
    rc = cuda_check(c, cudaMemcpyAsync(d_nloc, nloc.data(), sizeof(int) * 3 * nnew, cudaMemcpyHostToDevice, c->stream),
                    "remap locations");
  if (rc) return rc;
  Container &ob = c->md["base"];
  const long long cells = (long long)m.nx[0] * m.nx[1] * m.nx[2] * nnew;
  if (cells >= (1LL << 32)) {
    c->err = "adaptive mesh: more than 2^32 cells";
    return KMY_ERR_BAD_PARAM;
  }
  const dim3 rgrid(nblk(cells), unsigned(c->ncc + NPRIM));
  if (c->esz == 8)
    k_amr_remap<double><<<rgrid, kThreads, 0, c->stream>>>(
        mo, (const double *)ob.cc, nullptr, (const double *)c->prim, nnew, d_nlev, d_nloc, (double *)nb_ct.cc,
        nullptr, (double *)nprim, c->ncc, a.d_err);
  else
    k_amr_remap<float><<<rgrid, kThreads, 0, c->stream>>>(
        mo, (const float *)ob.cc, (const float *)ob.ener_lo, (const float *)c->prim, nnew, d_nlev, d_nloc,
        (float *)nb_ct.cc, (float *)nb_ct.ener_lo, (float *)nprim, c->ncc, a.d_err);
  c->launches++;
  if (c->prm.mhd) {
    const long long faces = (long long)(m.nx[0] + 1) * (m.nx[1] + 1) * (m.nx[2] + 1) * 3 * nnew;
    if (c->esz == 8)
      k_amr_remap_faces<double><<<nblk(faces), kThreads, 0, c->stream>>>(mo, (const double *)ob.fc, nnew, d_nlev,
                                                                         d_nloc, (double *)nb_ct.fc, a.d_err);
    else
      k_amr_remap_faces<float><<<nblk(faces), kThreads, 0, c->stream>>>(mo, (const float *)ob.fc, nnew, d_nlev,
                                                                        d_nloc, (float *)nb_ct.fc, a.d_err);
    c->launches++;
  }
  rc = cuda_check(c, cudaGetLastError(), "amr remap");
  if (!rc) rc = cuda_check(c, cudaStreamSynchronize(c->stream), "amr remap sync");
  if (rc) return rc;

  // release the old mesh's storage (stream ordered after the remap)
  for (auto &kv : c->md) {
    dfree(c, kv.second.cc);
    dfree(c, kv.second.ener_lo);
    dfree(c, kv.second.fc);
    dfree(c, kv.second.emf);
  }
  c->md.clear();
  dfree(c, c->prim);
  dfree(c, c->flux);
  c->flux = nullptr;
  if (c->prm.mhd) {
    // div B at the new block count (recomputed on the next last stage)
    dfree(c, c->divb);
    c->divb = nullptr;
    rc = dalloc(c, reinterpret_cast<void **>(&c->divb), 8 * n_new);
    if (rc) return rc;
  }
  dfree(c, d_nlev);
  dfree(c, d_nloc);
  a.lev = nlev;
  a.loc = nloc;
  a.cnt = ncnt;
  rc = amr_upload(c);
  if (rc) return rc;
  c->md["base"] = nb_ct;
  c->prim = nprim;
  const auto &nm = c->prm.stage_name;
  for (size_t s = 1; s + 1 < nm.size() && !rc; s++)
    if (!c->md.count(nm[s])) rc = make_container(c, nm[s]);
  if (!rc) rc = launch_amr_fill_ghosts(c, c->md["base"]);
  if (rc) return rc;
  *changed_out = true;
  return KMY_OK;
}

}  // namespace kmy

namespace kmy {

int amr_adopt_leaves(kmy_ctx *c) {
  c->amr.balanced = false;
  for (auto &kv : c->md) {
    dfree(c, kv.second.cc);
    dfree(c, kv.second.ener_lo);
    dfree(c, kv.second.fc);
    dfree(c, kv.second.emf);
  }
  c->md.clear();
  dfree(c, c->prim);
  c->prim = nullptr;
  dfree(c, c->flux);
  c->flux = nullptr;
  dfree(c, c->divb);
  c->divb = nullptr;
  int rc = amr_upload(c);
  if (rc) return rc;
  const size_t n = size_t(c->m.nb) * c->m.P;
  const auto &nm = c->prm.stage_name;
  for (size_t s = 0; s + 1 < nm.size() && !rc; s++)
    if (!c->md.count(nm[s])) rc = make_container(c, nm[s]);
  if (!rc) rc = dalloc(c, &c->prim, c->esz * NPRIM * n);
  if (!rc && c->prm.mhd) rc = dalloc(c, reinterpret_cast<void **>(&c->divb), 8 * n);
  return rc;
}

}  // namespace kmy

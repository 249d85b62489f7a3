// kmy_pgen.cu -- device problem generators.  Each sets density, velocity and
// pressure on the interior of "base" (and face B for CT) the way the
// reference's ProblemGenerator does; kmy_pgen then runs the dens_pres EOS
// initialisation and ConvertToConserved.
//
//   isentropic_vortex  src/problems/isentropic_vortex.hpp:31-51
//   sedov              src/problems/sedov.cpp:54-63, :75-103
//   blast              src/problems/mhd_blast.cpp:52-64 (no field)
//   kelvin_helmholtz   3D shear layer, v,w seeded per global cell (splitmix64)
//   orszag_tang        3D Orszag-Tang with face B from A_z (isentropic_vortex.cpp:150-174 pattern)
#include <cmath>
#include <string>

#include "../../include/kmy_hydro.h"
#include "kmy_internal.hpp"

namespace kmy {

enum Problem { P_VORTEX = 0, P_KH = 1, P_OT = 2, P_BLAST = 3, P_SEDOV = 4 };

struct PgenParams {
  int problem;
  int mhd;
  double gamma;
  double p[8];
  unsigned long long seed;
};

template <typename S>
__global__ void k_pgen_cells(MeshDesc m, PgenParams pp, S *cc, S *prim) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long per = (long long)m.nx[0] * m.nx[1] * m.nx[2];
  if (t >= per * m.nb) return;
  const int b = int(t / per);
  long long r = t - (long long)b * per;
  const int i = int(r % m.nx[0]);
  r /= m.nx[0];
  const int j = int(r % m.nx[1]);
  const int k = int(r / m.nx[1]);
  const int lx0 = blk_loc(m, b, 0), lx1 = blk_loc(m, b, 1), lx2 = blk_loc(m, b, 2);
  const long long gi = (long long)lx0 * m.nx[0] + i, gj = (long long)lx1 * m.nx[1] + j,
                  gk = (long long)lx2 * m.nx[2] + k;
  const double x = m.xmin[0] + (double(gi) + 0.5) * blk_dx(m, b, 0);
  const double y = m.xmin[1] + (double(gj) + 0.5) * blk_dx(m, b, 1);
  double dens = 1.0, v0 = 0.0, v1 = 0.0, v2 = 0.0, pres = 1.0;
  const double gamma = pp.gamma;
  if (pp.problem == P_VORTEX && pp.mhd) {
    // isentropic_vortex.hpp:75-100 (StateMHD); cell B comes from the faces
    const double pressure = pp.p[1], velx = pp.p[2], vely = pp.p[3], strength = pp.p[4],
                 mhd_strength = pp.p[5];
    const double r2 = x * x + y * y;
    const double dv = strength * exp(0.5 * (1.0 - r2)) / (2.0 * M_PI);
    const double ex = exp(1.0 - r2);
    dens = 1.0;
    pres = pressure + (mhd_strength * mhd_strength / (8.0 * M_PI * M_PI)) * (1.0 - r2) * ex -
           (strength * strength / (8.0 * M_PI * M_PI)) * ex;
    v0 = velx - y * dv;
    v1 = vely + x * dv;
  } else if (pp.problem == P_VORTEX) {
    const double density = pp.p[0], pressure = pp.p[1], velx = pp.p[2], vely = pp.p[3],
                 strength = pp.p[4];
    const double r2 = x * x + y * y;
    const double dv = strength * exp(0.5 * (1.0 - r2)) / (2.0 * M_PI);
    const double T = pressure / density -
                     (gamma - 1.0) * strength * strength * exp(1.0 - r2) / (8.0 * gamma * M_PI * M_PI);
    dens = pow(T, 1.0 / (gamma - 1.0));
    pres = T * dens;
    v0 = velx - y * dv;
    v1 = vely + x * dv;
  } else if (pp.problem == P_KH) {
    const double amp = pp.p[0];
    const bool inner = fabs(y - 0.5) < 0.25;
    dens = inner ? 2.0 : 1.0;
    v0 = inner ? 0.5 : -0.5;
    pres = 2.5;
    const unsigned long long gidx = ((unsigned long long)gk * (unsigned long long)m.mesh_nx[1] +
                                     (unsigned long long)gj) * (unsigned long long)m.mesh_nx[0] +
                                    (unsigned long long)gi;
    v1 = amp * (kh_uniform(pp.seed, gidx, 0) - 0.5);
    v2 = m.ndim > 2 ? amp * (kh_uniform(pp.seed, gidx, 1) - 0.5) : 0.0;
  } else if (pp.problem == P_OT) {
    dens = 25. / (36. * M_PI);
    pres = 5. / (12. * M_PI);
    v0 = -sin(2. * M_PI * y);
    v1 = sin(2. * M_PI * x);
  } else if (pp.problem == P_BLAST || pp.problem == P_SEDOV) {
    const double rr = sqrt(x * x + y * y);
    dens = pp.p[0];
    pres = rr <= pp.p[3] ? pp.p[2] : pp.p[1];
  }
  const long long NP = (long long)m.nb * m.P;
  const long long n = (long long)b * m.P +
                      ((long long)(k + m.g[2]) * m.np[1] + (j + m.g[1])) * m.np[0] + (i + m.g[0]);
  cc[n] = S(dens);
  prim[PVEL0 * NP + n] = S(v0);
  prim[PVEL1 * NP + n] = S(v1);
  prim[PVEL2 * NP + n] = S(v2);
  prim[PPRES * NP + n] = S(pres);
}

// Face B from the vector potential A_z of the Orszag-Tang problem:
// Bx = (A(xf, y+dy/2) - A(xf, y-dy/2))/dy, By = -(A(x+dx/2, yf) - A(x-dx/2, yf))/dx.
template <typename S>
__global__ void k_pgen_faces(MeshDesc m, PgenParams pp, S *fc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int n0 = m.nx[0] + 1, n1 = m.nx[1] + 1, n2 = m.nx[2] + (m.ndim > 2 ? 1 : 0);
  const long long per = (long long)n0 * n1 * n2;
  if (t >= per * m.nb) return;
  const int b = int(t / per);
  long long r = t - (long long)b * per;
  const int i = int(r % n0);
  r /= n0;
  const int j = int(r % n1);
  const int k = int(r / n1);
  const int lx0 = blk_loc(m, b, 0), lx1 = blk_loc(m, b, 1);
  const double dx0 = blk_dx(m, b, 0), dx1 = blk_dx(m, b, 1);
  const double xf = m.xmin[0] + double(lx0 * m.nx[0] + i) * dx0;
  const double yf = m.xmin[1] + double(lx1 * m.nx[1] + j) * dx1;
  const double xc = xf + 0.5 * dx0, yc = yf + 0.5 * dx1;
  const double B0 = 1.0 / sqrt(4.0 * M_PI);
  auto Az = [&](double X, double Y) {
    if (pp.problem == P_VORTEX)  // isentropic_vortex.hpp:140-144
      return pp.p[5] / (2. * M_PI) * exp(0.5 * (1.0 - (X * X + Y * Y)));
    if (pp.problem != P_OT) return 0.0;
    return B0 * (cos(4. * M_PI * X) / (4. * M_PI) + cos(2. * M_PI * Y) / (2. * M_PI));
  };
  const long long NF = (long long)m.nb * m.Pf;
  const long long o = (long long)b * m.Pf +
                      ((long long)(k + m.g[2]) * m.nf[1] + (j + m.g[1])) * m.nf[0] + (i + m.g[0]);
  fc[o] = S(1. / dx1 * (Az(xf, yc + 0.5 * dx1) - Az(xf, yc - 0.5 * dx1)));
  fc[NF + o] = S(-1. / dx0 * (Az(xc + 0.5 * dx0, yf) - Az(xc - 0.5 * dx0, yf)));
  if (m.ndim > 2) fc[2 * NF + o] = S(0);
}

int launch_pgen(kmy_ctx *c, const std::string &problem) {
  const Params &p = c->prm;
  PgenParams pp{};
  pp.gamma = p.gamma;
  if (problem == "isentropic_vortex") {
    pp.problem = P_VORTEX;
    pp.p[0] = p.real("isentropic_vortex/density", 1.0);
    pp.p[1] = p.real("isentropic_vortex/pressure", 1.0);
    pp.p[2] = p.real("isentropic_vortex/velx", 1.0);
    pp.p[3] = p.real("isentropic_vortex/vely", 1.0);
    pp.p[4] = p.real("isentropic_vortex/strength", 5.0);
    pp.p[5] = p.real("isentropic_vortex/mhd_strength", 1.0);
    pp.mhd = p.mhd ? 1 : 0;
  } else if (problem == "kelvin_helmholtz") {
    pp.problem = P_KH;
    pp.p[0] = p.real("kelvin_helmholtz/amplitude", 0.01);
    pp.seed = (unsigned long long)p.integer("kelvin_helmholtz/seed", 12345);
  } else if (problem == "orszag_tang") {
    pp.problem = P_OT;
  } else if (problem == "blast") {
    pp.problem = P_BLAST;
    pp.p[0] = p.real("blast/density", 1.0);
    pp.p[1] = p.real("blast/pressure", 0.1);
    pp.p[2] = p.real("blast/explosion_pressure", 10.0);
    pp.p[3] = p.real("blast/radius", 0.1);
  } else if (problem == "sedov") {
    pp.problem = P_SEDOV;
    const double E = p.real("sedov/energy", 1.0);
    const int nlev = p.integer("parthenon/mesh/numlevel", 1);
    const double dxs = c->m.dx[0] / std::pow(2.0, nlev - 1);
    const double radius = 3.5 * dxs;
    const double nu = 2.;
    pp.p[0] = p.real("sedov/density", 1.0);
    pp.p[1] = p.real("sedov/pressure", 1.0e-5);
    pp.p[2] = 3. * (p.gamma - 1) * E / ((nu + 1) * M_PI * std::pow(radius, nu));
    pp.p[3] = radius;
  } else {
    c->err = "unknown problem " + problem;
    return KMY_ERR_BAD_PARAM;
  }
  const MeshDesc &m = c->m;
  Container &b = c->md["base"];
  const long long n = (long long)m.nx[0] * m.nx[1] * m.nx[2] * m.nb;
  const unsigned grid = unsigned((n + 255) / 256);
  if (c->esz == 8)
    k_pgen_cells<double><<<grid, 256, 0, c->stream>>>(m, pp, (double *)b.cc, (double *)c->prim);
  else
    k_pgen_cells<float><<<grid, 256, 0, c->stream>>>(m, pp, (float *)b.cc, (float *)c->prim);
  c->launches++;
  if (c->prm.mhd) {
    const long long nf = (long long)(m.nx[0] + 1) * (m.nx[1] + 1) * (m.nx[2] + (m.ndim > 2)) * m.nb;
    const unsigned gf = unsigned((nf + 255) / 256);
    if (c->esz == 8)
      k_pgen_faces<double><<<gf, 256, 0, c->stream>>>(m, pp, (double *)b.fc);
    else
      k_pgen_faces<float><<<gf, 256, 0, c->stream>>>(m, pp, (float *)b.fc);
    c->launches++;
  }
  return cuda_check(c, cudaGetLastError(), "pgen");
}

}  // namespace kmy

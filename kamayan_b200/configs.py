"""Input decks of the standard workloads (Parthenon deck syntax).

``vortex_2d``    2D isentropic vortex, gamma 1.4, periodic [-5,5]^2, 128^2 in
                 4 blocks of 64^2 (2 ghosts), FP64, PLM(MC)+HLL, RK2, CFL 0.8, t=10.
``kh_3d``        3D Kelvin-Helmholtz, gamma 1.4, periodic unit cube, 256^3 in 512
                 blocks of 32^3 (3 ghosts), WENO-Z+HLLC, RK3, CFL 0.4, 200 steps.
``ot_3d``        3D Orszag-Tang with constrained transport, gamma 5/3, periodic unit
                 cube, 192^3 in 216 blocks of 32^3 (4 ghosts), PPM+HLL, RK2, CFL 0.3, t=0.5.
``blast_2d``     2D blast, gamma 5/3, [-0.5,0.5]^2, 128^2 in 16^2 blocks, PLM+HLLC,
                 RK2, t=0.2 (single-level form of the AMR workload).
``blast_2d_amr`` the same blast on an adaptive mesh: 3 levels, Loehner tagging on
                 density (refine 0.3, derefine 0.05).

Every builder takes keyword overrides for the mesh size so tests can run the
same physics on small meshes.
"""
from __future__ import annotations

from .deck import Deck


def _mesh(d: Deck, n: tuple, nb: tuple, xmin: tuple, xmax: tuple, bc: str, nghost: int) -> Deck:
    for i, ax in enumerate("123"):
        d.set("parthenon/mesh", f"nx{ax}", n[i])
        d.set("parthenon/mesh", f"x{ax}min", xmin[i])
        d.set("parthenon/mesh", f"x{ax}max", xmax[i])
        d.set("parthenon/mesh", f"ix{ax}_bc", bc)
        d.set("parthenon/mesh", f"ox{ax}_bc", bc)
        d.set("parthenon/meshblock", f"nx{ax}", nb[i])
    d.set("parthenon/mesh", "nghost", nghost)
    d.set("parthenon/mesh", "refinement", "none")
    return d


def vortex_2d(n: int = 128, nb: int = 64, recon: str = "plm", limiter: str = "mc",
              riemann: str = "hll", integrator: str = "rk2", nghost: int = 2,
              precision: str = "fp64", tlim: float = 10.0) -> Deck:
    d = Deck()
    _mesh(d, (n, n, 1), (nb, nb, 1), (-5.0, -5.0, -5.0), (5.0, 5.0, 5.0), "periodic", nghost)
    d.set("parthenon/time", "integrator", integrator)
    d.set("parthenon/time", "tlim", tlim)
    d.set("hydro", "reconstruction", recon)
    d.set("hydro", "slope_limiter", limiter)
    d.set("hydro", "riemann", riemann)
    d.set("hydro", "cfl", 0.8)
    d.set("eos", "mode_init", "dens_pres")
    d.set("material/single", "gamma", 1.4)
    d.set("isentropic_vortex", "density", 1.0)
    d.set("isentropic_vortex", "pressure", 1.0)
    d.set("isentropic_vortex", "velx", 1.0)
    d.set("isentropic_vortex", "vely", 1.0)
    d.set("isentropic_vortex", "strength", 5.0)
    d.set("kamayan_b200", "precision", precision)
    return d


def mhd_vortex_2d(n: int = 64, nb: int = 32, recon: str = "ppm", limiter: str = "mc",
                  riemann: str = "hll", nghost: int = 4, precision: str = "fp64",
                  tlim: float = 10.0) -> Deck:
    """The reference's CT vortex regression (tests/test_suites/mhd_vortex/mhd_vortex.py:37-55)."""
    d = vortex_2d(n=n, nb=nb, recon=recon, limiter=limiter, riemann=riemann, nghost=nghost,
                  precision=precision, tlim=tlim)
    d.set("physics", "MHD", "ct")
    d.set("isentropic_vortex", "strength", 1.0)
    d.set("isentropic_vortex", "mhd_strength", 1.0)
    return d


def kh_3d(n: int = 256, nb: int = 32, precision: str = "fp64", recon: str = "wenoz",
          riemann: str = "hllc", integrator: str = "rk3", nghost: int = 3, seed: int = 20240611,
          nlim: int = 200) -> Deck:
    d = Deck()
    _mesh(d, (n, n, n), (nb, nb, nb), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "periodic", nghost)
    d.set("parthenon/time", "integrator", integrator)
    d.set("parthenon/time", "nlim", nlim)
    d.set("hydro", "reconstruction", recon)
    d.set("hydro", "slope_limiter", "mc")
    d.set("hydro", "riemann", riemann)
    d.set("hydro", "cfl", 0.4)
    d.set("eos", "mode_init", "dens_pres")
    d.set("material/single", "gamma", 1.4)
    d.set("kelvin_helmholtz", "amplitude", 0.01)
    d.set("kelvin_helmholtz", "seed", seed)
    d.set("kamayan_b200", "precision", precision)
    return d


def ot_3d(n: int = 192, nb: int = 32, precision: str = "fp64", nghost: int = 4,
          tlim: float = 0.5) -> Deck:
    d = Deck()
    _mesh(d, (n, n, n), (nb, nb, nb), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), "periodic", nghost)
    d.set("parthenon/time", "integrator", "rk2")
    d.set("parthenon/time", "tlim", tlim)
    d.set("physics", "MHD", "ct")
    d.set("hydro", "reconstruction", "ppm")
    d.set("hydro", "slope_limiter", "mc")
    d.set("hydro", "riemann", "hll")
    d.set("hydro", "cfl", 0.3)
    d.set("eos", "mode_init", "dens_pres")
    d.set("material/single", "gamma", 5.0 / 3.0)
    d.set("kamayan_b200", "precision", precision)
    return d


def blast_2d(n: int = 128, nb: int = 16, precision: str = "fp64", bc: str = "outflow",
             recon: str = "plm", riemann: str = "hllc", nghost: int = 2, tlim: float = 0.2) -> Deck:
    d = Deck()
    _mesh(d, (n, n, 1), (nb, nb, 1), (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5), bc, nghost)
    d.set("parthenon/time", "integrator", "rk2")
    d.set("parthenon/time", "tlim", tlim)
    d.set("hydro", "reconstruction", recon)
    d.set("hydro", "slope_limiter", "mc")
    d.set("hydro", "riemann", riemann)
    d.set("hydro", "cfl", 0.8)
    d.set("eos", "mode_init", "dens_pres")
    d.set("material/single", "gamma", 5.0 / 3.0)
    d.set("blast", "density", 1.0)
    d.set("blast", "pressure", 0.1)
    d.set("blast", "explosion_pressure", 10.0)
    d.set("blast", "radius", 0.1)
    d.set("kamayan_b200", "precision", precision)
    return d


def blast_2d_amr(n: int = 128, nb: int = 16, precision: str = "fp64", numlevel: int = 3,
                 refine_tol: float = 0.3, derefine_tol: float = 0.05, tlim: float = 0.2,
                 derefine_count: int = 10, field: str = "dens") -> Deck:
    """The AMR workload: ``blast_2d`` on an adaptive mesh with Loehner tagging on density."""
    d = blast_2d(n=n, nb=nb, precision=precision, tlim=tlim)
    d.set("parthenon/mesh", "refinement", "adaptive")
    d.set("parthenon/mesh", "numlevel", numlevel)
    d.set("parthenon/mesh", "derefine_count", derefine_count)
    d.set("kamayan/refinement0", "field", field)
    d.set("kamayan/refinement0", "method", "loehner")
    d.set("kamayan/refinement0", "refine_tol", refine_tol)
    d.set("kamayan/refinement0", "derefine_tol", derefine_tol)
    d.set("kamayan/refinement0", "max_level", numlevel - 1)
    return d


def mhd_vortex_2d_amr(n: int = 64, nb: int = 8, numlevel: int = 2, refine_tol: float = 0.02,
                      field: str = "pres", derefine_count: int = 2, precision: str = "fp64") -> Deck:
    """The CT vortex on an adaptive mesh: Loehner tagging on pressure refines the
    vortex core, and the core's motion refines and derefines blocks as it goes."""
    d = mhd_vortex_2d(n=n, nb=nb, precision=precision)
    d.set("parthenon/mesh", "refinement", "adaptive")
    d.set("parthenon/mesh", "numlevel", numlevel)
    d.set("parthenon/mesh", "derefine_count", derefine_count)
    d.set("kamayan/refinement0", "field", field)
    d.set("kamayan/refinement0", "refine_tol", refine_tol)
    d.set("kamayan/refinement0", "derefine_tol", refine_tol / 4)
    return d

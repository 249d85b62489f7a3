"""The oracle against the reference's own known answers (CPU only).

Pins the oracle with the reference's unit and regression tests:
reconstruction exactness and symmetry (test_reconstruction.cpp:159-194), the
ideal-gas EOS (test_eos.cpp:55-85), the per-method density-L1 thresholds of
the vortex at 64^2, t=10 (tests/test_suites/reconstruction/reconstruction.py:128-135)
and the WENO-Z/RK2 convergence slope > 1.5
(tests/test_suites/isentropic_vortex/isentropic_vortex.py:13-60).
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from kamayan_b200 import configs

GOLD = Path(__file__).resolve().parent / "golden"


def ulps(a: float, b: float) -> int:
    ia = np.array([a]).view(np.int64)[0]
    ib = np.array([b]).view(np.int64)[0]
    return abs(int(ia) - int(ib))


def test_reconstruction_polynomial_exactness(oracle_mod):
    for case in json.loads((GOLD / "reconstruction_kat.json").read_text()):
        vm, vp = oracle_mod.reconstruct(case["reconstruction"], case["slope_limiter"], case["stencil"])
        assert abs((vm - case["exact_minus"]) / case["exact_minus"]) < case["rel_tol"], case
        assert abs((vp - case["exact_plus"]) / case["exact_plus"]) < case["rel_tol"], case


def test_reconstruction_left_right_symmetry(oracle_mod):
    for case in json.loads((GOLD / "reconstruction_kat.json").read_text()):
        fwd = case["tanh_stencil"]
        rev = list(reversed(fwd))
        vm1, vp1 = oracle_mod.reconstruct(case["reconstruction"], case["slope_limiter"], fwd)
        vm2, vp2 = oracle_mod.reconstruct(case["reconstruction"], case["slope_limiter"], rev)
        assert ulps(vm1, vp2) <= case["symmetry_ulps"], case["reconstruction"]
        assert ulps(vp1, vm2) <= case["symmetry_ulps"], case["reconstruction"]


def test_fog_copies_cell_value(oracle_mod):
    vm, vp = oracle_mod.reconstruct("fog", "minmod", [1, 2, 3.5, 4, 5])
    assert vm == vp == 3.5


def test_eos_ideal_gas(oracle_mod):
    k = json.loads((GOLD / "eos_kat.json").read_text())
    out = oracle_mod.eos(k["gamma"], k["Abar"], "pres", k["rho"], 0.0, 0.0, k["pres"], 0.0)
    assert abs(out["sie"] - k["eint"]) < k["eint_tol"]
    back = oracle_mod.eos(k["gamma"], k["Abar"], "ener", k["rho"], 0.0, out["sie"], -1.0, 0.0)
    assert back["pres"] == k["pres_back_exact"]
    # bulk modulus of an ideal gas is gamma * P
    assert back["bmod"] == pytest.approx(k["gamma"] * k["pres"], rel=1e-15)


def test_riemann_uniform_state_is_physical_flux(oracle_mod):
    # equal left/right states: HLL and HLLC return the exact Euler flux
    rho, u, v, w, p, gam = 1.3, 0.4, -0.2, 0.1, 2.0, 1.4
    eint = p / ((gam - 1) * rho)
    V = [rho, u, v, w, p, gam * p, eint]
    E = rho * eint + 0.5 * rho * (u * u + v * v + w * w)
    exact = [rho * u, rho * u * u + p, rho * u * v, rho * u * w, (E + p) * u]
    for solver in ("hll", "hllc"):
        f = oracle_mod.riemann(solver, False, 0, V, V)
        np.testing.assert_allclose(f, exact, rtol=1e-14, atol=1e-15)


def test_riemann_mirror_symmetry(oracle_mod):
    # mirrored states give a mass flux of opposite sign
    L = [1.0, 0.3, 0.1, 0.0, 1.0, 1.4, 2.5]
    R = [0.5, -0.2, 0.0, 0.2, 0.3, 0.42, 1.5]
    for solver in ("hll", "hllc"):
        f = oracle_mod.riemann(solver, False, 0, L, R)
        Lm = [R[0], -R[1], R[2], R[3], R[4], R[5], R[6]]
        Rm = [L[0], -L[1], L[2], L[3], L[4], L[5], L[6]]
        g = oracle_mod.riemann(solver, False, 0, Lm, Rm)
        assert f[0] == pytest.approx(-g[0], rel=1e-13)
        assert f[1] == pytest.approx(g[1], rel=1e-13)


THRESHOLDS = [("fog", "minmod", 0.3), ("plm", "minmod", 0.08), ("plm", "mc", 0.02),
              ("plm", "van_leer", 0.03), ("ppm", "minmod", 0.02), ("ppm", "mc", 0.015),
              ("wenoz", "minmod", 0.005)]


@pytest.mark.parametrize("recon,limiter,max_error", THRESHOLDS)
def test_vortex_density_l1_thresholds(oracle_mod, recon, limiter, max_error):
    deck = configs.vortex_2d(n=64, nb=32, recon=recon, limiter=limiter, riemann="hll", nghost=3)
    s = oracle_mod.OracleSim(deck.text())
    s.pgen("isentropic_vortex")
    s.evolve(10.0)
    assert s.time["time"] == pytest.approx(10.0, abs=1e-12)
    err = s.vortex_error("dens")
    assert err < max_error and np.isfinite(err)


def test_vortex_convergence_wenoz(oracle_mod):
    res = [32, 64]
    errs = []
    for n in res:
        deck = configs.vortex_2d(n=n, nb=n // 2, recon="wenoz", nghost=3)
        s = oracle_mod.OracleSim(deck.text())
        s.pgen("isentropic_vortex")
        s.evolve(10.0)
        errs.append(s.vortex_error("dens"))
    slopes = [-math.log(errs[i] / errs[i - 1]) / math.log(res[i] / res[i - 1]) for i in range(1, len(res))]
    assert min(slopes) > 1.5, slopes


def test_mhd_vortex_ct_threshold(oracle_mod):
    """CT vortex: PPM-MC, HLL, RK2, 64^2, t=10; magx L1 < 0.05 (mhd_vortex.py:25-27,298-299)
    and div B at round-off."""
    s = oracle_mod.OracleSim(configs.mhd_vortex_2d().text())
    s.pgen("isentropic_vortex")
    s.evolve(10.0)
    err = s.vortex_error("magc", 0)
    assert err < 0.05 and np.isfinite(err)
    assert np.abs(s.interior(s.get("divb"))).max() < 1e-10


def test_oracle_thread_count_independent(oracle_mod):
    # the oracle's OpenMP block loops must not change a single bit
    import os
    import subprocess
    import sys

    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from oracle import oracle as O\n"
        "from kamayan_b200 import configs\n"
        "d = configs.kh_3d(n=16, nb=8)\n"
        "s = O.OracleSim(d.text()); s.pgen('kelvin_helmholtz'); s.step(); s.step()\n"
        "import hashlib; print(hashlib.sha256(s.get('ener').tobytes()).hexdigest())\n"
    ) % str(Path(__file__).resolve().parent.parent)
    outs = []
    for nt in ("1", "4"):
        env = dict(os.environ, OMP_NUM_THREADS=nt)
        outs.append(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True,
                                   text=True, check=True).stdout.strip())
    assert outs[0] == outs[1]

"""FP32 bulk path: accuracy against FP64, conservation, import path (GPU).

Bar: density L1 of the FP32 run relative to the FP64 run <= 1e-5 on the
3D WENO-Z/HLLC Kelvin-Helmholtz workload (and the other methods).
"""
import numpy as np
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs

from parity import rel_l1

pytestmark = pytest.mark.gpu

L1_FP32 = 1e-5


def _pair(deck32, deck64, problem, nsteps, path="fused"):
    out = []
    for d in (deck32, deck64):
        s = K.Solver(d)
        s.set_path(path)
        s.pgen(problem)
        for _ in range(nsteps):
            s.step()
        out.append(s)
    return out


@pytest.mark.parametrize("path", ["fused", "tasks"])
def test_kh3d_fp32_vs_fp64(kmy_lib, path):
    s32, s64 = _pair(configs.kh_3d(n=32, nb=16, precision="fp32"),
                     configs.kh_3d(n=32, nb=16, precision="fp64"), "kelvin_helmholtz", 10, path)
    for var, c in [("dens", 0), ("momentum", 0), ("ener", 0)]:
        err = rel_l1(s32.interior(s32.export(var, c)), s64.interior(s64.export(var, c)))
        assert err <= L1_FP32, (var, err)
    t32, t64 = s32.time, s64.time
    assert np.isfinite(t32["dt"]) and t32["dt"] > 0
    assert abs(t32["time"] - t64["time"]) <= 1e-5 * t64["time"]


@pytest.mark.parametrize("path", ["fused", "tasks"])
def test_orszag_tang_fp32_vs_fp64(kmy_lib, path):
    """3D Orszag-Tang with constrained transport, FP32 bulk against FP64."""
    s32, s64 = _pair(configs.ot_3d(n=32, nb=16, precision="fp32"),
                     configs.ot_3d(n=32, nb=16, precision="fp64"), "orszag_tang", 5, path)
    for var, c in [("dens", 0), ("momentum", 0), ("momentum", 1), ("ener", 0), ("magc", 0), ("magc", 1)]:
        err = rel_l1(s32.interior(s32.export(var, c)), s64.interior(s64.export(var, c)))
        assert err <= L1_FP32, (var, c, err)
    # div B of the FP32 face field, evaluated in FP64
    assert np.abs(s32.interior(s32.export("divb"))).max() < 1e-4


@pytest.mark.parametrize("recon,riemann", [("plm", "hll"), ("ppm", "hllc"), ("wenoz", "hllc")])
def test_vortex2d_fp32_vs_fp64(kmy_lib, recon, riemann):
    s32, s64 = _pair(configs.vortex_2d(n=64, nb=32, recon=recon, riemann=riemann, nghost=3,
                                       precision="fp32"),
                     configs.vortex_2d(n=64, nb=32, recon=recon, riemann=riemann, nghost=3,
                                       precision="fp64"), "isentropic_vortex", 20)
    err = rel_l1(s32.interior(s32.export("dens")), s64.interior(s64.export("dens")))
    assert err <= L1_FP32, err


def test_conservation_periodic(kmy_lib):
    for prec, tol in (("fp64", 1e-13), ("fp32", 1e-6)):
        s = K.Solver(configs.kh_3d(n=32, nb=16, precision=prec))
        s.pgen("kelvin_helmholtz")
        m0 = s.conserved_sums()
        for _ in range(5):
            s.step()
        m1 = s.conserved_sums()
        # mass and total energy are conserved by the flux form on a periodic mesh
        assert abs(m1[0] - m0[0]) <= tol * abs(m0[0]), prec
        assert abs(m1[4] - m0[4]) <= tol * abs(m0[4]), prec


def test_fp32_import_then_step(kmy_lib):
    src = K.Solver(configs.kh_3d(n=32, nb=16, precision="fp64"))
    src.pgen("kelvin_helmholtz")
    s = K.Solver(configs.kh_3d(n=32, nb=16, precision="fp32"))
    for v, c in [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0),
                 ("velocity", 0), ("velocity", 1), ("velocity", 2), ("pres", 0),
                 ("bulk modulus", 0), ("eint", 0), ("temp", 0)]:
        s.import_(v, src.export(v, c), c)
    s.finalize_import()
    for _ in range(3):
        s.step()
        src.step()
    assert rel_l1(s.interior(s.export("dens")), src.interior(src.export("dens"))) <= L1_FP32
    # energy round-trips through the hi/lo split to FP64 accuracy at import
    s2 = K.Solver(configs.kh_3d(n=32, nb=16, precision="fp32"))
    e = src.export("ener")
    s2.import_("ener", e)
    back = s2.export("ener", container="base")
    assert rel_l1(s2.interior(back), src.interior(e)) <= 1e-14

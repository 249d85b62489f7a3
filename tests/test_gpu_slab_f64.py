"""The z-streamed stage in FP64 (kmy_slab.cuh, 8-row tiles) on the GPU.

* its face ghosts equal what Parthenon's boundary exchange puts there, bit for
  bit, for periodic, outflow, reflecting and mixed boundaries;
* it matches the oracle to 1e-12 relative L1 after one step for every
  reconstruction and both Riemann solvers, and to 1e-10 over several steps for
  every integrator, non-periodic boundaries and uneven blocks;
* it matches the FP64 brick stage to 1e-12;
* whole runs through kmy_evolve's CUDA graphs give the same bits as one step
  per call, and its bounded wait reports a timeout without faulting.
"""
import numpy as np
import pytest

import kamayan_b200 as K

from parity import CONS, compare, rel_l1, run_pair
from test_gpu_slab import BCS, kh, pulled_face_ghosts, run

pytestmark = pytest.mark.gpu

TOL_1STEP = 1e-12
TOL_NSTEP = 1e-10


def kh64(**kw):
    kw.setdefault("kernel", "slab")
    return kh(precision="fp64", **kw)


def _check(res: dict, tol: float):
    bad = {k: v for k, v in res.items() if not (v <= tol)}
    assert not bad, f"relative L1 above {tol}: {bad}"


def test_fp64_default_is_the_slab_on_large_meshes(kmy_lib):
    # 192^3: 864 work items of 8 rows; 64^3: 32, too few to fill the GPU
    assert K.Solver(kh64(kernel="auto", n=192)).stage_kernel == "slab8"
    assert K.Solver(kh64(kernel="auto")).stage_kernel == "brick"


@pytest.mark.parametrize("bcname", list(BCS))
def test_slab64_face_ghosts_match_exchange(kmy_lib, bcname):
    bc = BCS[bcname]
    s = K.Solver(kh64(bc=bc))
    s._bcs = [(a.replace("reflecting", "reflect"), b.replace("reflecting", "reflect")) for a, b in bc]
    s.pgen("kelvin_helmholtz")
    s.rk_stage(1)
    for var, c in CONS:
        arr = s.export(var, c, container="1")
        flip = c if var == "momentum" else None
        mask, want = pulled_face_ghosts(s, arr, flip)
        np.testing.assert_array_equal(arr[mask], want[mask], err_msg=f"{bcname} {var}{c}")


@pytest.mark.parametrize("recon,riemann,limiter", [
    ("wenoz", "hllc", "mc"), ("wenoz", "hll", "mc"), ("ppm", "hllc", "mc"), ("ppm", "hll", "minmod"),
    ("plm", "hllc", "van_leer"), ("plm", "hll", "mc"), ("fog", "hllc", "mc")])
def test_slab64_one_step_vs_oracle(kmy_lib, oracle_mod, recon, riemann, limiter):
    d = kh64(recon=recon, riemann=riemann)
    d.set("hydro", "slope_limiter", limiter)
    o, s, _ = run_pair(d, "kelvin_helmholtz", 1, "fused")
    assert s.stage_kernel == "slab8"
    _check(compare(o, s), TOL_1STEP)


@pytest.mark.parametrize("integrator", ["rk1", "rk2", "rk3"])
def test_slab64_integrators_vs_oracle(kmy_lib, oracle_mod, integrator):
    o, s, _ = run_pair(kh64(integrator=integrator), "kelvin_helmholtz", 4, "fused")
    _check(compare(o, s), TOL_NSTEP)


@pytest.mark.parametrize("bcname", ["outflow", "reflect", "mixed"])
def test_slab64_boundaries_vs_oracle(kmy_lib, oracle_mod, bcname):
    o, s, _ = run_pair(kh64(bc=BCS[bcname]), "kelvin_helmholtz", 4, "fused")
    _check(compare(o, s), TOL_NSTEP)


def test_slab64_uneven_blocks_vs_oracle(kmy_lib, oracle_mod):
    """Blocks of 32 x 48 x 34 (six row tiles, an odd number of plane pairs)."""
    o, s, _ = run_pair(kh64(dims=((64, 96, 68), (32, 48, 34))), "kelvin_helmholtz", 3, "fused")
    _check(compare(o, s), TOL_NSTEP)


def test_slab64_vs_brick(kmy_lib):
    a, b = run(kh64(), 6), run(kh64(kernel="brick"), 6)
    assert a.stage_kernel == "slab8" and b.stage_kernel == "brick"
    for var, c in CONS:
        err = rel_l1(a.interior(a.export(var, c)), b.interior(b.export(var, c)))
        assert err <= TOL_1STEP, (var, c, err)


def test_slab64_evolve_graph_matches_steps(kmy_lib):
    a = K.Solver(kh64(nlim=30))
    a.pgen("kelvin_helmholtz")
    n = a.evolve(1e30, 12)
    b = run(kh64(nlim=30), n)
    for var, c in CONS:
        np.testing.assert_array_equal(a.export(var, c), b.export(var, c))


def test_slab64_stage_wait_runs_out(kmy_lib):
    s = K.Solver(kh64())
    s.pgen("kelvin_helmholtz")
    s.set_fault("stage_wait")
    with pytest.raises(K.KmyError) as e:
        s.step()
    assert e.value.code == 4  # KMY_ERR_TIMEOUT

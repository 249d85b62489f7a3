"""Constrained transport on the GPU against the oracle, through the task
path and the fused stage.

Covers the CT pieces of the hot path: face-field Riemann override, widened
flux bounds (the fused stage's ghost-layer flux copies), edge EMFs, the
Stokes face update, the face->cell average in PreparePrimitive and div B in
FP64.
"""
import numpy as np
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs

from parity import compare, run_pair

pytestmark = pytest.mark.gpu


def _check(res: dict, tol: float):
    bad = {k: v for k, v in res.items() if not (v <= tol)}
    assert not bad, f"relative L1 above {tol}: {bad}"


PATHS = ["tasks", "fused"]


@pytest.mark.parametrize("path", PATHS)
def test_mhd_vortex_2d_ct(kmy_lib, oracle_mod, path):
    deck = configs.mhd_vortex_2d(n=32, nb=16)
    o, s, _ = run_pair(deck, "isentropic_vortex", 1, path, mhd=True)
    _check(compare(o, s, mhd=True, prims=True), 1e-12)


@pytest.mark.parametrize("path", PATHS)
def test_mhd_vortex_2d_ct_multistep(kmy_lib, oracle_mod, path):
    deck = configs.mhd_vortex_2d(n=32, nb=16)
    o, s, _ = run_pair(deck, "isentropic_vortex", 6, path, mhd=True)
    _check(compare(o, s, mhd=True), 1e-10)


@pytest.mark.parametrize("path", PATHS)
def test_orszag_tang_3d_ct(kmy_lib, oracle_mod, path):
    # 12^3 blocks: the fused stage's 8^3 bricks are partial at every block's
    # high edge
    deck = configs.ot_3d(n=24, nb=12)
    o, s, _ = run_pair(deck, "orszag_tang", 1, path, mhd=True)
    _check(compare(o, s, mhd=True, prims=True), 1e-12)
    o2, s2, _ = run_pair(deck, "orszag_tang", 4, path, mhd=True)
    _check(compare(o2, s2, mhd=True), 1e-10)


def test_orszag_tang_divb_fp64(kmy_lib):
    s = K.Solver(configs.ot_3d(n=32, nb=16))
    s.pgen("orszag_tang")
    for _ in range(5):
        s.step()
    divb = s.interior(s.export("divb"))
    assert np.sqrt(np.mean(divb ** 2)) < 1e-10
    assert np.abs(divb).max() < 1e-10


def test_mhd_vortex_gpu_threshold(kmy_lib):
    """The reference's CT vortex bar (magx L1 < 0.05 at t=10) on the GPU path."""
    s = K.Solver(configs.mhd_vortex_2d())
    s.pgen("isentropic_vortex")
    s.evolve(10.0)
    assert s.time["time"] == pytest.approx(10.0, abs=1e-12)
    assert s.vortex_error("magc", 0) < 0.05


@pytest.mark.parametrize("path", PATHS)
def test_ct_outflow_boundaries(kmy_lib, oracle_mod, path):
    # outflow boundaries: the fused stage's ghost-layer flux copies take the
    # boundary row itself (periodic meshes never reach that branch)
    deck = configs.mhd_vortex_2d(n=32, nb=16)
    for ax in "12":
        deck.set("parthenon/mesh", f"ix{ax}_bc", "outflow").set("parthenon/mesh", f"ox{ax}_bc", "outflow")
    o, s, _ = run_pair(deck, "isentropic_vortex", 4, path, mhd=True)
    _check(compare(o, s, mhd=True), 1e-10)
    deck3 = configs.ot_3d(n=24, nb=12)
    deck3.set("parthenon/mesh", "ix1_bc", "outflow").set("parthenon/mesh", "ox1_bc", "outflow")
    o3, s3, _ = run_pair(deck3, "orszag_tang", 3, path, mhd=True)
    _check(compare(o3, s3, mhd=True), 1e-10)


def test_ct_rk1_runs_the_task_kernels(kmy_lib, oracle_mod):
    # rk1 is outside the fused CT stage: steps go through the per-task kernels
    deck = configs.mhd_vortex_2d(n=32, nb=16)
    deck.set("parthenon/time", "integrator", "rk1")
    o, s, _ = run_pair(deck, "isentropic_vortex", 3, "fused", mhd=True)
    _check(compare(o, s, mhd=True), 1e-10)

"""The z-streamed stage with constrained transport (FP32, kmy_slab.cuh with
MHD) on the GPU.

* it matches the FP64 run (itself oracle-parity-tested) to the FP32 bar of
  1e-5 relative L1 per conserved variable and face field, and the FP32 brick
  stage to the same bar, with 8- and 16-row tiles, periodic and outflow
  boundaries;
* the cell pass writes the field's face ghosts as Parthenon's exchange would
  fill them, bit for bit, so the next stage stages current ghost zones;
* div B stays at FP32 rounding.
"""
import numpy as np
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs

from parity import rel_l1
from test_gpu_slab import pulled_face_ghosts

pytestmark = pytest.mark.gpu

L1_FP32 = 1e-5
FIELDS = [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0),
          ("magc", 0), ("magc", 1), ("magc", 2)]


def ot(precision="fp32", kernel="slab", rows=None, outflow=False, n=64):
    d = configs.ot_3d(n=n, nb=32, precision=precision)
    d.set("kamayan_b200", "stage_kernel", kernel)
    if rows is not None:
        d.set("kamayan_b200", "slab_rows", rows)
    if outflow:
        d.set("parthenon/mesh", "ix1_bc", "outflow").set("parthenon/mesh", "ox1_bc", "outflow")
    return d


def run(deck, nsteps):
    s = K.Solver(deck)
    s.pgen("orszag_tang")
    for _ in range(nsteps):
        s.step()
    return s


def close(a, b, tol):
    for var, c in FIELDS:
        err = rel_l1(a.interior(a.export(var, c)), b.interior(b.export(var, c)))
        assert err <= tol, (var, c, err)
    for c in range(3):
        err = rel_l1(a.export("mag", c), b.export("mag", c))
        assert err <= tol, ("mag", c, err)


def test_default_kernel_is_the_slab_on_large_meshes(kmy_lib):
    # 192^3: 432 work items of 16 rows; 64^3: 16, too few to fill the GPU
    assert K.Solver(ot(kernel="auto", n=192)).stage_kernel == "slab16"
    assert K.Solver(ot(kernel="auto")).stage_kernel == "brick"
    assert K.Solver(ot(precision="fp64", kernel="auto", n=192)).stage_kernel == "brick"


@pytest.mark.parametrize("rows", ["8", "16"])
@pytest.mark.parametrize("outflow", [False, True])
def test_ct_slab_vs_fp64(kmy_lib, rows, outflow):
    s32 = run(ot(rows=rows, outflow=outflow), 5)
    assert s32.stage_kernel == f"slab{rows}"
    s64 = run(ot(precision="fp64", kernel="auto", outflow=outflow), 5)
    close(s32, s64, L1_FP32)
    assert abs(s32.time["time"] - s64.time["time"]) <= 1e-5 * s64.time["time"]
    assert np.abs(s32.interior(s32.export("divb"))).max() < 1e-4


def test_ct_slab_vs_brick(kmy_lib):
    a, b = run(ot(), 5), run(ot(kernel="brick"), 5)
    assert a.stage_kernel == "slab16" and b.stage_kernel == "brick"
    close(a, b, L1_FP32)


@pytest.mark.parametrize("outflow", [False, True])
def test_ct_slab_field_ghosts_match_exchange(kmy_lib, outflow):
    s = K.Solver(ot(outflow=outflow))
    s._bcs = [("outflow", "outflow") if (outflow and d == 0) else ("periodic", "periodic") for d in range(3)]
    s.pgen("orszag_tang")
    s.step()  # RK2: the first stage's output stays in container "1"
    for c in range(3):
        arr = s.export("magc", c, container="1")
        mask, want = pulled_face_ghosts(s, arr)
        np.testing.assert_array_equal(arr[mask], want[mask], err_msg=f"magc{c}")
    for var, c in FIELDS[:5]:
        arr = s.export(var, c, container="1")
        mask, want = pulled_face_ghosts(s, arr)
        np.testing.assert_array_equal(arr[mask], want[mask], err_msg=f"{var}{c}")


def test_ct_slab_evolve_graph_matches_steps(kmy_lib):
    a = K.Solver(ot())
    a.pgen("orszag_tang")
    n = a.evolve(1e30, 6)
    b = run(ot(), n)
    for var, c in FIELDS:
        np.testing.assert_array_equal(a.export(var, c), b.export(var, c))

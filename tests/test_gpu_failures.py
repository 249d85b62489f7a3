"""Failure detection (GPU): every failure is made on the host or by a wait
that runs out; nothing faults, traps or hangs the GPU.

* a NaN density imported into a healthy state: the step returns
  KMY_ERR_NONFINITE (the device dt controller sees the non-finite CFL
  estimate; the reference's analogue is its dt checks,
  src/driver/kamayan_driver.cpp:43-54), on the brick and z-streamed paths;
* Parthenon's dt sanity limits: a dt below dt_min for dt_min_cycle_limit
  cycles, or above dt_max, ends the run with KMY_ERR_DT_RANGE;
* the z-streamed stage's bounded wait for its staged plane pairs runs out
  (its barrier expects bytes no load delivers): the step returns
  KMY_ERR_TIMEOUT and the CUDA context stays usable;
* the serving loop: one poisoned request among healthy ones fails alone,
  the others give the same bits as when they run alone; a request larger
  than the HBM budget is refused at submission.
"""
import math

import numpy as np
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs

pytestmark = pytest.mark.gpu

CONS = [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0)]


def _poison(s):
    d = s.export("dens")
    g = s.info.nghost
    d[0, g + 1, g + 2, g + 3] = float("nan")
    s.import_("dens", d)
    s.finalize_import()


def _slab(deck):
    deck.set("kamayan_b200", "stage_kernel", "slab")
    return deck


@pytest.mark.parametrize("deck", [configs.kh_3d(n=32, nb=16),                           # FP64 brick
                                  _slab(configs.kh_3d(n=64, nb=32, precision="fp32"))],  # FP32 z-streamed
                         ids=["fp64_brick", "fp32_slab"])
def test_nan_density_returns_nonfinite(kmy_lib, deck):
    s = K.Solver(deck)
    s.pgen("kelvin_helmholtz")
    s.step()
    _poison(s)
    with pytest.raises(K.KmyError) as e:
        for _ in range(3):
            s.step()
    assert e.value.code == 3  # KMY_ERR_NONFINITE


def test_nan_density_stops_evolve(kmy_lib):
    s = K.Solver(configs.kh_3d(n=32, nb=16, nlim=50))
    s.pgen("kelvin_helmholtz")
    _poison(s)
    with pytest.raises(K.KmyError) as e:
        s.evolve(1e30, 20)
    assert e.value.code == 3


def test_dt_below_dt_min_for_the_cycle_limit(kmy_lib):
    d = configs.kh_3d(n=32, nb=16)
    d.set("parthenon/time", "dt_min", 1.0)  # far above the CFL dt
    d.set("parthenon/time", "dt_min_cycle_limit", 3)
    s = K.Solver(d)
    s.pgen("kelvin_helmholtz")
    s.step()
    s.step()  # two cycles below dt_min: still running
    with pytest.raises(K.KmyError) as e:
        s.step()
    assert e.value.code == 7  # KMY_ERR_DT_RANGE


def test_dt_above_dt_max(kmy_lib):
    d = configs.kh_3d(n=32, nb=16)
    d.set("parthenon/time", "dt_max", 1e-9)
    s = K.Solver(d)
    s.pgen("kelvin_helmholtz")
    with pytest.raises(K.KmyError) as e:
        s.evolve(1e30, 10)
    assert e.value.code == 7


def test_stage_wait_runs_out(kmy_lib):
    deck = configs.kh_3d(n=64, nb=32, precision="fp32")
    deck.set("kamayan_b200", "stage_kernel", "slab")
    s = K.Solver(deck)
    s.pgen("kelvin_helmholtz")
    assert s.stage_kernel.startswith("slab")
    s.set_fault("stage_wait")
    with pytest.raises(K.KmyError) as e:
        s.step()
    assert e.value.code == 4  # KMY_ERR_TIMEOUT
    s.close()
    # the CUDA context is still usable: a new solve runs and matches a second one
    runs = []
    for _ in range(2):
        t = K.Solver(deck)
        t.pgen("kelvin_helmholtz")
        for _ in range(3):
            t.step()
        runs.append(t.export("dens"))
        t.close()
    np.testing.assert_array_equal(runs[0], runs[1])


def test_fault_hook_rejects_unknown_and_inapplicable(kmy_lib):
    s = K.Solver(configs.kh_3d(n=32, nb=16))  # 16^3 blocks: no z-streamed stage
    with pytest.raises(K.KmyError):
        s.set_fault("stage_wait")
    with pytest.raises(K.KmyError):
        s.set_fault("no_such_fault")


NSTEPS = 6


def _alone(deck, problem):
    s = K.Solver(deck)
    s.pgen(problem)
    for _ in range(NSTEPS):
        s.step()
    out = [s.export(v, c) for v, c in CONS]
    shape = s.cell_shape
    s.close()
    return out, shape


def test_server_poisoned_request_fails_alone(kmy_lib):
    healthy = [(configs.vortex_2d(n=64, nb=32), "isentropic_vortex"),
               (configs.kh_3d(n=32, nb=16, precision="fp32"), "kelvin_helmholtz"),
               (configs.blast_2d(n=64, nb=16), "blast")]
    bad = configs.blast_2d(n=64, nb=16)
    bad.set("blast", "explosion_pressure", float("nan"))
    srv = K.Server(hbm_fraction=0.5)
    ids = [srv.submit(d, p, NSTEPS) for d, p in healthy[:2]]
    bad_id = srv.submit(bad, "blast", NSTEPS)
    ids.append(srv.submit(*healthy[2], NSTEPS))
    done = {}
    for _ in range(1000):
        active, queued = srv.tick()
        for rid, secs, st in srv.poll():
            done[rid] = st
        if active == 0 and queued == 0:
            break
    for rid, secs, st in srv.poll():
        done[rid] = st
    assert done[bad_id] == 3  # KMY_ERR_NONFINITE
    for rid, (d, p) in zip(ids, healthy):
        assert done[rid] == 0
        want, shape = _alone(d, p)
        for (v, c), w in zip(CONS, want):
            np.testing.assert_array_equal(srv.export(rid, v, shape, c), w, err_msg=f"{p} {v}{c}")
        srv.release(rid)


def test_server_refuses_a_request_above_the_budget(kmy_lib):
    srv = K.Server(hbm_fraction=1e-7)  # a budget of a few kilobytes
    with pytest.raises(K.KmyError) as e:
        srv.submit(configs.kh_3d(n=32, nb=16), "kelvin_helmholtz", 5)
    assert e.value.code == 2  # KMY_ERR_OOM
    st = srv.stats
    assert st["queued"] == 0 and st["active"] == 0
    assert not math.isnan(st["budget"]) and st["budget"] > 0

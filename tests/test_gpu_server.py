"""Serving loop: continuous batching of independent solves (GPU).

Each request's result must be bit-identical whether it runs alone (one
context, kmy_step) or inside the batched persistent launches with other
requests of mixed sizes, methods and precisions, admitted at different ticks.
"""
import numpy as np
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs

pytestmark = pytest.mark.gpu

NSTEPS = 8
CONS = [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0)]


def _mix():
    return [
        (configs.vortex_2d(n=64, nb=32, recon="plm", riemann="hll"), "isentropic_vortex"),
        (configs.vortex_2d(n=32, nb=16, recon="plm", riemann="hll"), "isentropic_vortex"),
        (configs.vortex_2d(n=32, nb=16, recon="ppm", riemann="hllc", nghost=3, precision="fp32"),
         "isentropic_vortex"),
        (configs.kh_3d(n=32, nb=16), "kelvin_helmholtz"),
        (configs.kh_3d(n=16, nb=8, precision="fp32"), "kelvin_helmholtz"),
        (configs.blast_2d(n=64, nb=16, precision="fp32"), "blast"),
        (configs.blast_2d(n=32, nb=16, recon="wenoz", nghost=3, bc="reflect"), "blast"),
    ]


def _alone(deck, problem):
    s = K.Solver(deck)
    s.pgen(problem)
    for _ in range(NSTEPS):
        s.step()
    out = [s.export(v, c) for v, c in CONS]
    shape = s.cell_shape
    s.close()
    return out, shape


def _drain(srv, limit=10000):
    done = {}
    for _ in range(limit):
        active, queued = srv.tick()
        for rid, secs, st in srv.poll():
            done[rid] = (secs, st)
        if active == 0 and queued == 0:
            break
    for rid, secs, st in srv.poll():
        done[rid] = (secs, st)
    return done


def test_results_identical_alone_and_in_the_mix(kmy_lib):
    mix = _mix()
    srv = K.Server(hbm_fraction=0.5)
    ids = []
    # half now, half after a few ticks: continuous admission
    for deck, prob in mix[: len(mix) // 2]:
        ids.append(srv.submit(deck, prob, NSTEPS))
    for _ in range(3):
        srv.tick()
    for deck, prob in mix[len(mix) // 2:]:
        ids.append(srv.submit(deck, prob, NSTEPS))
    done = _drain(srv)
    assert set(done) == set(ids)
    assert all(st == 0 for _, st in done.values())
    for rid, (deck, prob) in zip(ids, mix):
        ref, shape = _alone(deck, prob)
        for (v, c), r in zip(CONS, ref):
            got = srv.export(rid, v, shape, c)
            assert np.array_equal(got, r), (deck.get("hydro", "reconstruction"), v, c)
        srv.release(rid)
    st = srv.stats
    assert st["finished"] == len(mix) and st["bytes_in_use"] == 0
    srv.close()


def test_admission_respects_budget(kmy_lib):
    import torch

    deck = configs.kh_3d(n=32, nb=16)
    # one request holds 3 containers x 5 + 7 primitive words on 8 x 22^3 cells
    per_request = 8 * 22 ** 3 * (3 * 5 + 7) * 8
    free = torch.cuda.mem_get_info()[0]
    srv = K.Server(hbm_fraction=2.5 * per_request / free)  # room for two at a time
    budget = srv.stats["budget"]
    ids = []
    for _ in range(12):
        try:
            ids.append(srv.submit(deck, "kelvin_helmholtz", 4))
        except K.KmyError as e:
            pytest.skip(f"budget too small for one request: {e}")
    peak = 0
    done = {}
    for _ in range(10000):
        active, queued = srv.tick()
        st = srv.stats
        assert st["bytes_in_use"] <= budget
        peak = max(peak, active)
        for rid, secs, s in srv.poll():
            done[rid] = s
            srv.release(rid)
        if active == 0 and queued == 0:
            break
    assert sorted(done) == sorted(ids)
    assert 1 <= peak <= 2
    srv.close()


def test_server_rejects_unsupported(kmy_lib):
    srv = K.Server(hbm_fraction=0.1)
    with pytest.raises(K.KmyError):
        srv.submit(configs.ot_3d(n=24, nb=12), "orszag_tang", 2)   # CT runs on the task path
    with pytest.raises(K.KmyError):
        srv.submit(configs.vortex_2d(n=32, nb=16, integrator="rk1"), "isentropic_vortex", 2)
    srv.close()


def test_fused_rk1_matches_tasks(kmy_lib):
    """rk1 updates base in place; the fused stage writes a scratch container."""
    out = []
    for path in ("fused", "tasks"):
        s = K.Solver(configs.kh_3d(n=32, nb=16, integrator="rk1"))
        s.set_path(path)
        s.pgen("kelvin_helmholtz")
        for _ in range(4):
            s.step()
        out.append(s.interior(s.export("dens")))
    assert np.abs(out[0] - out[1]).max() <= 1e-12 * np.abs(out[1]).max()

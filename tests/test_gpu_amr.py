"""Adaptive mesh on the GPU against the CPU oracle (GPU required).

The oracle restates Parthenon's block tree (refine, 2:1 balance with corners,
derefine after derefine_count tags, Morton order) and kamayan's refinement
operators; the library runs the same steps with its device kernels.  Checks:
identical leaf lists after the initial refinement and after every step,
bit-identical ghost cells from the level exchange on identical interiors,
state parity in relative L1 after several steps, and conservation across
fine/coarse faces (flux correction).
"""
import numpy as np
import pytest

from kamayan_b200 import configs

from parity import CONS, PRIMS, compare

pytestmark = pytest.mark.gpu

TOL_NSTEP = 1e-10


def _pair(deck, problem="blast"):
    from kamayan_b200 import Solver
    from oracle.oracle import OracleSim

    text = deck.text()
    o = OracleSim(text)
    o.pgen(problem)
    s = Solver(text)
    s.set_path("tasks")
    s.pgen(problem)
    return o, s


def _same_blocks(o, s):
    lo, co = o.blocks()
    ls, cs = s.blocks()
    assert len(lo) == len(ls), f"block count {len(ls)} != oracle {len(lo)}"
    assert np.array_equal(lo, ls), "levels differ"
    assert np.array_equal(co, cs), "locations differ"
    return len(lo)


def test_initial_refinement_on_pressure(kmy_lib, oracle_mod):
    # the pressure jump of the blast refines at set-up (initial refinement loop)
    deck = configs.blast_2d_amr(n=64, nb=8, field="pres")
    o, s = _pair(deck)
    nb = _same_blocks(o, s)
    lev, _ = s.blocks()
    assert nb > 64 and lev.max() == 2
    res = compare(o, s, prims=True)
    assert all(v <= 1e-13 for v in res.values()), res
    assert abs(s.time["dt"] - o.time["dt"]) <= 1e-14 * o.time["dt"]


@pytest.mark.parametrize("bc", ["outflow", "reflecting", "periodic"])
def test_level_exchange_bit_identical(kmy_lib, oracle_mod, bc):
    # identical interiors on an identical 3-level mesh: every ghost cell (copy,
    # restriction of finer leaves, minmod prolongation, and the corners where
    # a prolongation's coarse neighbour is itself restricted or prolongated)
    # matches bit for bit, mirrored components included
    deck = configs.blast_2d_amr(n=64, nb=8, field="pres")
    for ax in "12":
        deck.set("parthenon/mesh", f"ix{ax}_bc", bc).set("parthenon/mesh", f"ox{ax}_bc", bc)
        if bc != "outflow":
            # the blast (centred on the origin) near the low corner, so the
            # refined levels reach the boundary and its mapped ghost cells
            deck.set("parthenon/mesh", f"x{ax}min", -0.125).set("parthenon/mesh", f"x{ax}max", 0.875)
    o, s = _pair(deck)
    _same_blocks(o, s)
    for var, c in CONS + PRIMS:
        s.import_(var, o.get(var, c), c)
    s.finalize_import()
    for var, c in CONS + PRIMS:
        a, b = s.export(var, c), o.get(var, c)
        assert np.array_equal(a, b), f"{var}{c}: max |diff| {np.abs(a - b).max()}"


@pytest.mark.parametrize("field", ["dens", "pres"])
def test_blast_steps_blocks_and_state(kmy_lib, oracle_mod, field):
    # refinement and derefinement during the run (derefine_count 2 so blocks
    # coarsen behind the shock within the test's steps)
    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2, field=field)
    o, s = _pair(deck)
    _same_blocks(o, s)
    counts = []
    for _ in range(40):
        s.set_dt(o.time["dt"])
        o.step()
        s.step()
        counts.append(_same_blocks(o, s))
        assert abs(s.time["dt"] - o.time["dt"]) <= 1e-12 * o.time["dt"]
    assert max(counts) > counts[0] or counts[0] > 64, "the mesh never refined"
    res = compare(o, s, prims=True)
    bad = {k: v for k, v in res.items() if not v <= TOL_NSTEP}
    assert not bad, bad


def test_derefinement_happens(kmy_lib, oracle_mod):
    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2)
    o, s = _pair(deck)
    counts = []
    for _ in range(60):
        s.set_dt(o.time["dt"])
        o.step()
        s.step()
        counts.append(_same_blocks(o, s))
    assert any(b < a for a, b in zip(counts, counts[1:])), counts


def test_conservation_across_levels(kmy_lib, oracle_mod):
    # periodic box: total mass and energy change only by rounding when fine
    # fluxes replace coarse ones at level boundaries
    deck = configs.blast_2d_amr(n=64, nb=8, field="pres")
    for ax in "12":
        deck.set("parthenon/mesh", f"ix{ax}_bc", "periodic").set("parthenon/mesh", f"ox{ax}_bc", "periodic")
    from kamayan_b200 import Solver

    s = Solver(deck.text())
    s.pgen("blast")
    lev, _ = s.blocks()
    assert lev.max() == 2
    m0 = s.conserved_sums()
    for _ in range(20):
        s.step()
    m1 = s.conserved_sums()
    for v in (0, 4):
        assert abs(m1[v] - m0[v]) <= 1e-13 * abs(m0[v]), (v, m0[v], m1[v])


def test_fp32_amr_close_to_fp64(kmy_lib):
    from kamayan_b200 import Solver

    out = {}
    for prec in ("fp64", "fp32"):
        deck = configs.blast_2d_amr(n=64, nb=8, field="pres", precision=prec)
        s = Solver(deck.text())
        s.pgen("blast")
        for _ in range(10):
            s.step()
        out[prec] = (s.blocks(), s.interior(s.export("dens")))
    (l64, c64), d64 = out["fp64"]
    (l32, c32), d32 = out["fp32"]
    assert np.array_equal(l64, l32) and np.array_equal(c64, c32)
    assert np.abs(d32 - d64).sum() / np.abs(d64).sum() <= 1e-5


def test_fused_stage_rejects_adaptive_mesh(kmy_lib):
    from kamayan_b200 import KmyError, Solver

    s = Solver(configs.blast_2d_amr(n=64, nb=8).text())
    s.pgen("blast")
    with pytest.raises(KmyError):
        s.rk_stage(1)


def test_server_refuses_adaptive_deck(kmy_lib):
    # the serving loop batches fixed meshes; an adaptive deck is refused at submit
    from kamayan_b200 import KmyError, Server

    srv = Server()
    try:
        with pytest.raises(KmyError):
            srv.submit(configs.blast_2d_amr(n=64, nb=8), "blast", 4)
    finally:
        srv.close()


def test_two_criteria_take_the_larger_tag(kmy_lib, oracle_mod):
    # <kamayan/refinement0> on density and <kamayan/refinement1> on pressure:
    # a block's tag is the larger of the two criteria's
    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2)
    deck.set("kamayan/refinement1", "field", "pres")
    deck.set("kamayan/refinement1", "refine_tol", 0.5)
    deck.set("kamayan/refinement1", "derefine_tol", 0.1)
    deck.set("kamayan/refinement1", "max_level", 1)
    o, s = _pair(deck)
    _same_blocks(o, s)
    for _ in range(30):
        s.set_dt(o.time["dt"])
        o.step()
        s.step()
        _same_blocks(o, s)
    res = compare(o, s)
    assert all(v <= TOL_NSTEP for v in res.values()), res


def test_zone_cycles_count_each_step_on_its_mesh(kmy_lib):
    # the zone-cycle counter adds each step's interior cells before its
    # remesh, through kmy_step and through kmy_evolve alike
    from kamayan_b200 import Solver

    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2)
    s = Solver(deck.text())
    s.set_path("tasks")
    s.pgen("blast")
    assert s.zone_cycles == 0
    per_block = 8 * 8
    expect, counts = 0, set()
    for _ in range(60):  # derefinement within 60 steps: test_derefinement_happens
        counts.add(s.nblocks)
        expect += s.nblocks * per_block
        s.step()
    assert s.zone_cycles == expect
    assert len(counts) > 1, "the mesh never changed"
    n0, z0 = s.time["ncycle"], s.zone_cycles
    nb = s.nblocks
    s.evolve(1e30, 1)
    assert s.time["ncycle"] == n0 + 1 and s.zone_cycles == z0 + nb * per_block


def test_evolve_graph_matches_steps(kmy_lib):
    # kmy_evolve replays each adaptive step's stages from a CUDA graph
    # (captured again after every remesh); kmy_step launches them one by one.
    # Same meshes, same bits.
    from kamayan_b200 import Solver

    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2)
    sa, sb = Solver(deck.text()), Solver(deck.text())
    for s in (sa, sb):
        s.set_path("tasks")
        s.pgen("blast")
    for _ in range(60):
        sa.step()
    sb.evolve(1e30, 30)
    r30 = sb.graph_replays
    sb.evolve(1e30, 30)
    assert sa.time == sb.time and sa.time["ncycle"] == 60
    # the steps replayed their captured graphs, also on meshes after a remesh
    assert r30 > 0 and sb.graph_replays > r30
    la, ca = sa.blocks()
    lb, cb = sb.blocks()
    assert np.array_equal(la, lb) and np.array_equal(ca, cb)
    for var, c in CONS + PRIMS:
        a, b = sa.export(var, c), sb.export(var, c)
        assert np.array_equal(a, b), f"{var}{c}: max |diff| {np.abs(a - b).max()}"
    assert sa.zone_cycles == sb.zone_cycles


def test_evolve_to_tlim_matches_steps(kmy_lib):
    # kmy_evolve queues each next step before it reads the current step's tags
    # (a speculative step, undone when the mesh changes or the run ends); to an
    # end time it gives what stepping one at a time gives, and it counts the
    # steps' device time
    from kamayan_b200 import Solver

    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2)
    probe = Solver(deck.text())
    probe.set_path("tasks")
    probe.pgen("blast")
    probe.evolve(1e30, 45)
    tlim = probe.time["time"] * 0.97  # the last step is clamped to land on tlim
    probe.close()
    sa, sb = Solver(deck.text()), Solver(deck.text())
    for s in (sa, sb):
        s.set_path("tasks")
        s.pgen("blast")
    while sa.time["time"] < tlim:
        sa.evolve(tlim, 1)
    sb.evolve(tlim)
    assert sb.time == sa.time and sb.time["time"] == tlim
    la, ca = sa.blocks()
    lb, cb = sb.blocks()
    assert np.array_equal(la, lb) and np.array_equal(ca, cb)
    for var, c in CONS + PRIMS:
        a, b = sa.export(var, c), sb.export(var, c)
        assert np.array_equal(a, b), f"{var}{c}: max |diff| {np.abs(a - b).max()}"
    assert sa.zone_cycles == sb.zone_cycles
    assert sb.evolve_device_ms > 0.0

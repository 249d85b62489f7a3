"""Restart files: a solve saved mid-run and resumed in a new context ends in
the same bits as the solve that kept running (GPU required)."""
import numpy as np
import pytest

from kamayan_b200 import configs

pytestmark = pytest.mark.gpu


def _run(deck, problem, before, after, path, tmp_path):
    from kamayan_b200 import Solver

    a = Solver(deck.text())
    a.set_path(path)
    a.pgen(problem)
    for _ in range(before):
        a.step()
    f = tmp_path / "state.rst"
    a.save_restart(f)
    for _ in range(after):
        a.step()
    b = Solver.from_restart(f)
    for _ in range(after):
        b.step()
    return a, b


def _same(a, b, names):
    assert a.time == b.time
    for var, c in names:
        x, y = a.export(var, c), b.export(var, c)
        assert np.array_equal(x, y), f"{var}{c}: max |diff| {np.abs(x - y).max()}"


CONS = [("dens", 0), ("momentum", 0), ("momentum", 1), ("ener", 0)]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_restart_fused_kh(kmy_lib, tmp_path, precision):
    deck = configs.kh_3d(n=32, nb=16, precision=precision)
    a, b = _run(deck, "kelvin_helmholtz", 3, 3, "fused", tmp_path)
    _same(a, b, CONS)


def test_restart_ct_tasks(kmy_lib, tmp_path):
    deck = configs.mhd_vortex_2d(n=64, nb=32)
    a, b = _run(deck, "isentropic_vortex", 4, 4, "tasks", tmp_path)
    _same(a, b, CONS + [("mag", 0), ("mag", 1), ("magc", 0)])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_restart_ct_fused(kmy_lib, tmp_path, precision):
    # the fused CT stage resumes from the saved primitives, faces and clock
    deck = configs.ot_3d(n=24, nb=12, precision=precision)
    a, b = _run(deck, "orszag_tang", 3, 3, "fused", tmp_path)
    _same(a, b, CONS + [("mag", 0), ("mag", 2), ("magc", 1)])


def test_restart_adaptive_mesh(kmy_lib, tmp_path):
    deck = configs.blast_2d_amr(n=64, nb=8, derefine_count=2)
    a, b = _run(deck, "blast", 20, 20, "tasks", tmp_path)
    la, ca = a.blocks()
    lb, cb = b.blocks()
    assert np.array_equal(la, lb) and np.array_equal(ca, cb)
    _same(a, b, CONS)


def test_restart_rejects_other_files(kmy_lib, tmp_path):
    from kamayan_b200 import KmyError, Solver

    bad = tmp_path / "not_a_restart"
    bad.write_bytes(b"hello world, not a restart file")
    with pytest.raises(KmyError):
        Solver.from_restart(bad)

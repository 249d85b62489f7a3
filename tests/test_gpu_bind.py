"""The boundary on caller-owned device memory (GPU).

The reference's slots read and write the MeshData they are handed
(src/kamayan/unit.hpp:56-76, src/grid/grid.hpp:133-135).  Here the caller
allocates the containers' arrays (torch tensors stand in for a framework's
device memory), binds them (kmy_bind_container, kmy_bind_primitives), writes
the state into them itself, and the per-task slots update them in place:

* one RK3 step through kmy_task_stage on bound arrays matches the oracle to
  1e-12, read straight from the caller's tensors;
* the fused and z-streamed paths on a bound "base" give the same bits as on
  the context's own arrays (rk3, and rk1 whose scratch output is copied back);
* misaligned, mis-sized and adaptive-mesh bindings are refused.
"""
import numpy as np
import pytest

import kamayan_b200 as K
from kamayan_b200 import configs

from parity import CONS, PRIMS, rel_l1

pytestmark = pytest.mark.gpu


def _torch():
    import torch

    return torch


def _bind_all(s, names):
    torch = _torch()
    inf = s.info
    shape = (inf.nblocks, *reversed(list(inf.ncells_pad)))
    dt = torch.float64 if inf.precision == 64 else torch.float32
    bufs = {}
    for name in names:
        cons = torch.zeros((inf.ncons, *shape), dtype=dt, device="cuda")
        lo = torch.zeros(shape, dtype=torch.float32, device="cuda") if inf.precision == 32 else None
        s.bind_container(name, cons.data_ptr(), cons.numel() * cons.element_size(),
                         lo.data_ptr() if lo is not None else 0, lo.numel() * 4 if lo is not None else 0)
        bufs[name] = (cons, lo)
    prim = torch.zeros((7, *shape), dtype=dt, device="cuda")
    s.bind_primitives(prim.data_ptr(), prim.numel() * prim.element_size())
    return bufs, prim


def test_task_stages_on_bound_arrays_match_oracle(kmy_lib, oracle_mod):
    torch = _torch()
    deck = configs.kh_3d(n=32, nb=16)  # FP64, RK3: containers base, 1, 2 and dUdt
    o = oracle_mod.OracleSim(deck.text())
    o.pgen("kelvin_helmholtz")
    s = K.Solver(deck)
    bufs, prim = _bind_all(s, ["base", "1", "2", "dUdt"])
    base = bufs["base"][0]
    # the caller writes the state into its own arrays
    for v, (var, c) in enumerate(CONS):
        base[v].copy_(torch.from_numpy(o.get(var, c)))
    torch.cuda.synchronize()
    s.finalize_import()
    dt = o.time["dt"]
    s.set_dt(dt)
    before = base.data_ptr()
    for stage in (1, 2, 3):
        s.task_stage(stage, dt)
    s.end_step()
    o.step()
    s.sync()
    assert base.data_ptr() == before
    got = base.cpu().numpy()
    for v, (var, c) in enumerate(CONS):
        err = rel_l1(o.interior(got[v]), o.interior(o.get(var, c)))
        assert err <= 1e-12, (var, c, err)
    # the primitives of the step's result, in the caller's primitive array
    pr = prim.cpu().numpy()
    for k, (var, c) in enumerate(PRIMS):
        err = rel_l1(o.interior(pr[k]), o.interior(o.get(var, c)))
        assert err <= 1e-12, (var, c, err)


@pytest.mark.parametrize("precision,integrator", [("fp32", "rk3"), ("fp64", "rk3"), ("fp64", "rk1"),
                                                  ("fp32", "rk1")])
def test_fused_steps_on_bound_base_same_bits(kmy_lib, precision, integrator):
    torch = _torch()
    deck = configs.kh_3d(n=64, nb=32, precision=precision, integrator=integrator)
    ref = K.Solver(deck)
    ref.pgen("kelvin_helmholtz")
    state = [ref.export(var, c) for var, c in CONS]
    # the context's own arrays, state imported through the C ABI
    own = K.Solver(deck)
    for (var, c), a in zip(CONS, state):
        own.import_(var, a, c)
    own.finalize_import()
    # the caller's arrays, the same state written by the caller
    s = K.Solver(deck)
    bufs, _ = _bind_all(s, ["base"])
    cons, lo = bufs["base"]
    for v, a in enumerate(state):
        cons[v].copy_(torch.from_numpy(a).to(cons.dtype))
    if lo is not None:
        e64 = torch.from_numpy(state[4])
        lo.copy_((e64 - e64.to(torch.float32).to(torch.float64)).to(torch.float32))
    torch.cuda.synchronize()
    s.finalize_import()
    for _ in range(4):
        own.step()
        s.step()
    s.sync()
    got = cons.cpu().numpy().astype(np.float64)
    if lo is not None:
        got[4] += lo.cpu().numpy().astype(np.float64)
    for v, (var, c) in enumerate(CONS):
        np.testing.assert_array_equal(s.interior(got[v]), own.interior(own.export(var, c)),
                                      err_msg=f"{precision} {integrator} {var}{c}")


def test_bind_rejects_bad_arrays(kmy_lib):
    torch = _torch()
    s = K.Solver(configs.kh_3d(n=32, nb=16))
    inf = s.info
    n = inf.ncons * inf.nblocks * int(np.prod(list(inf.ncells_pad)))
    t = torch.zeros(n + 8, dtype=torch.float64, device="cuda")
    with pytest.raises(K.KmyError):
        s.bind_container("base", t.data_ptr(), (n - 1) * 8)  # wrong size
    with pytest.raises(K.KmyError):
        s.bind_container("base", t.data_ptr() + 8, n * 8)  # not 16-byte aligned
    with pytest.raises(K.KmyError):
        s.bind_container("no such container", t.data_ptr(), n * 8)
    a = K.Solver(configs.blast_2d_amr(n=32, nb=16, numlevel=2))
    ai = a.info
    m = ai.ncons * ai.nblocks * int(np.prod(list(ai.ncells_pad)))
    u = torch.zeros(m, dtype=torch.float64, device="cuda")
    with pytest.raises(K.KmyError):
        a.bind_container("base", u.data_ptr(), m * 8)

"""Helpers that run the CUDA library and the CPU oracle on the same state.

The oracle generates the initial condition; the identical arrays are imported
into the CUDA library through the C ABI, so both start bit-identical.  Both
then step with the same dt and the interior states are compared per
conserved variable in relative L1.
"""
from __future__ import annotations

import numpy as np

CONS = [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0)]
PRIMS = [("velocity", 0), ("velocity", 1), ("velocity", 2), ("pres", 0), ("bulk modulus", 0),
         ("eint", 0), ("temp", 0)]
MHD_CELL = [("magc", 0), ("magc", 1), ("magc", 2)]


def rel_l1(a: np.ndarray, b: np.ndarray) -> float:
    den = np.abs(b).sum()
    num = np.abs(a - b).sum()
    if den == 0.0:
        return float(num)
    return float(num / den)


def transfer_state(o, s, mhd: bool = False) -> None:
    """Copy the oracle's base container and primitives into the solver."""
    for var, c in CONS + PRIMS + (MHD_CELL if mhd else []):
        s.import_(var, o.get(var, c), c)
    if mhd:
        for c in range(3):
            s.import_("mag", o.get("mag", c), c)
    s.finalize_import()


def compare(o, s, mhd: bool = False, prims: bool = False, container: str = "base") -> dict:
    out = {}
    names = CONS + (MHD_CELL if mhd else []) + (PRIMS if prims else [])
    for var, c in names:
        a = s.interior(s.export(var, c, container))
        b = o.interior(o.get(var, c, container))
        out[f"{var}{c}"] = rel_l1(a, b)
    if mhd:
        for c in range(3):
            out[f"mag{c}"] = rel_l1(s.export("mag", c, container), o.get("mag", c, container))
    return out


def run_pair(deck, problem: str, nsteps: int, path: str = "fused", mhd: bool = False):
    """Step oracle and solver nsteps times with the oracle's dt; return both."""
    from kamayan_b200 import Solver
    from oracle.oracle import OracleSim

    text = deck.text()
    o = OracleSim(text)
    o.pgen(problem)
    s = Solver(text)
    s.set_path(path)
    transfer_state(o, s, mhd)
    dts = []
    for _ in range(nsteps):
        dt = o.time["dt"]
        s.set_dt(dt)
        o.step()
        s.step()
        dts.append((dt, s.time["dt"], o.time["dt"]))
    return o, s, dts

"""The serving workload: a stream of independent solve requests.

Request i is drawn from numpy's generator seeded with base + i:
  size      uniform over {64^2, 128^2, 256^2, 64^3, 128^3}
  problem   isentropic vortex (strength ~ U[1,5]) or blast (pressure ratio
            log-uniform on [10, 1e4], radius ~ U[0.05, 0.15])
  method    PLM/HLL, PPM/HLLC or WENO-Z/HLLC
  precision FP32 or FP64
and runs for a fixed number of steps (100 by default).  ``run_stream`` feeds
the requests to a ``Server`` at their arrival times and records each
request's time to solution (arrival to completion).
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from . import configs
from .deck import Deck

SIZES = [(64, 2), (128, 2), (256, 2), (64, 3), (128, 3)]
METHODS = [("plm", "hll", 2), ("ppm", "hllc", 3), ("wenoz", "hllc", 3)]


@dataclass
class Request:
    index: int
    deck: Deck
    problem: str
    cells: int
    label: str


def make_request(index: int, base_seed: int = 1000) -> Request:
    rng = np.random.default_rng(base_seed + index)
    n, ndim = SIZES[rng.integers(len(SIZES))]
    recon, riemann, ng = METHODS[rng.integers(len(METHODS))]
    precision = "fp32" if rng.integers(2) == 0 else "fp64"
    vortex = rng.integers(2) == 0
    nb = 32
    if vortex:
        d = configs.vortex_2d(n=n, nb=nb, recon=recon, limiter="mc", riemann=riemann, nghost=ng,
                              precision=precision)
        d.set("isentropic_vortex", "strength", float(rng.uniform(1.0, 5.0)))
        problem = "isentropic_vortex"
    else:
        d = configs.blast_2d(n=n, nb=nb, recon=recon, riemann=riemann, nghost=ng,
                             precision=precision)
        ratio = float(10.0 ** rng.uniform(1.0, 4.0))
        d.set("blast", "explosion_pressure", ratio * 0.1)
        d.set("blast", "radius", float(rng.uniform(0.05, 0.15)))
        problem = "blast"
    if ndim == 3:
        lo, hi = (-5.0, 5.0) if vortex else (-0.5, 0.5)
        d.set("parthenon/mesh", "nx3", n).set("parthenon/meshblock", "nx3", nb)
        d.set("parthenon/mesh", "x3min", lo).set("parthenon/mesh", "x3max", hi)
    d.set("parthenon/time", "integrator", "rk2")
    return Request(index, d, problem, n ** ndim,
                   f"{problem} {n}^{ndim} {recon}/{riemann} {precision}")


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs), q)) if xs else None


def run_stream(requests, nsteps: int, arrivals=None, hbm_fraction: float = 0.7, graphs: bool = True,
               device: int = 0) -> dict:
    """Serve `requests` arriving at `arrivals` (seconds; None = all at t=0)."""
    from . import Server

    srv = Server(device=device, hbm_fraction=hbm_fraction, graphs=graphs)
    order = sorted(range(len(requests)), key=lambda k: 0.0 if arrivals is None else arrivals[k])
    arr = [0.0 if arrivals is None else float(arrivals[k]) for k in range(len(requests))]
    id_of = {}
    tts = {}
    nxt = 0
    t0 = time.perf_counter()
    work = 0.0
    while len(tts) < len(requests):
        now = time.perf_counter() - t0
        while nxt < len(order) and arr[order[nxt]] <= now:
            k = order[nxt]
            id_of[srv.submit(requests[k].deck, requests[k].problem, nsteps)] = k
            nxt += 1
        st = srv.stats
        if st["active"] == 0 and st["queued"] == 0 and nxt < len(order):
            # idle until the next arrival (with every request submitted, tick on:
            # the tick reports what is left)
            time.sleep(max(0.0, min(0.002, arr[order[nxt]] - now)))
            continue
        srv.tick()
        t_now = time.perf_counter() - t0
        for rid, _secs, status in srv.poll():
            k = id_of[rid]
            if status != 0:
                raise RuntimeError(f"request {k} ({requests[k].label}) failed with status {status}")
            tts[k] = t_now - arr[k]
            work += requests[k].cells * nsteps
            srv.release(rid)
    elapsed = time.perf_counter() - t0 - (min(arr) if arr else 0.0)
    stats = srv.stats
    srv.close()
    lat = [tts[k] for k in range(len(requests))]
    return {
        "requests": len(requests), "steps_each": nsteps, "elapsed_s": elapsed,
        "cell_updates_per_s": work / elapsed, "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99),
        "mean_s": float(np.mean(lat)), "ticks": int(stats["ticks"]), "launches": int(stats["launches"]),
    }


def run_sequential(requests, nsteps: int, device: int = 0) -> dict:
    """Each request alone, one after another (one context per solve, kmy_step per step)."""
    from . import Solver

    work = 0.0
    t0 = time.perf_counter()
    for r in requests:
        s = Solver(r.deck, device=device)
        s.pgen(r.problem)
        for _ in range(nsteps):
            s.step()
        s.close()
        work += r.cells * nsteps
    el = time.perf_counter() - t0
    return {"requests": len(requests), "elapsed_s": el, "cell_updates_per_s": work / el}


def poisson_arrivals(n: int, rate_per_s: float, seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))

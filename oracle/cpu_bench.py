"""Time the CPU oracle on a bounded sample of a workload (test/bench infrastructure).

Runs as its own process (``python -m oracle.cpu_bench``) so the oracle's
OpenMP runtime never shares a process with CUDA or torch.  Prints one JSON
object: cell-updates/s over the timed steps, the thread count, the CPU model,
the build and the sample.  ``--build native`` times the host-tuned build
(-O3 -march=native, compiled on this machine first); ``parity`` the portable
parity build.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

from kamayan_b200 import configs  # noqa: E402
from oracle import oracle  # noqa: E402


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="kh_3d")
    ap.add_argument("--n", type=int, default=128, help="cells per dimension of the sample mesh")
    ap.add_argument("--nb", type=int, default=32)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--min-seconds", type=float, default=0.0, help="keep stepping until this long")
    ap.add_argument("--max-steps", type=int, default=1000)
    ap.add_argument("--build", choices=["native", "parity"], default="native")
    a = ap.parse_args()
    threads = a.threads or len(os.sched_getaffinity(0))
    os.environ["OMP_NUM_THREADS"] = str(threads)
    oracle.use_native = a.build == "native"
    if a.workload == "kh_3d":
        deck, prob = configs.kh_3d(n=a.n, nb=a.nb), "kelvin_helmholtz"
    elif a.workload == "vortex_2d":
        deck, prob = configs.vortex_2d(n=a.n, nb=a.nb), "isentropic_vortex"
    elif a.workload == "ot_3d":
        deck, prob = configs.ot_3d(n=a.n, nb=a.nb), "orszag_tang"
    elif a.workload == "blast_2d_amr":
        deck, prob = configs.blast_2d_amr(n=a.n, nb=a.nb), "blast"
    else:
        raise SystemExit(f"unknown workload {a.workload}")
    s = oracle.OracleSim(deck.text())
    s.pgen(prob)
    for _ in range(a.warmup):
        s.step()
    ndim = s.info["ndim"]
    block_cells = s.info["nx1"] * s.info["nx2"] * s.info["nx3"]
    t0 = time.perf_counter()
    done = updates = 0
    while done < a.steps or (time.perf_counter() - t0 < a.min_seconds and done < a.max_steps):
        s.refresh()  # the block count changes on an adaptive mesh
        updates += s.info["nb"] * block_cells
        s.step()
        done += 1
    el = time.perf_counter() - t0
    a.steps = done
    cells = a.n ** ndim
    print(json.dumps({"value": updates / el, "unit": "cell-updates/s", "seconds": el,
                      "steps": a.steps, "cells": cells, "threads": threads, "cpu": cpu_model(),
                      "build": ("-O3 -march=native -ffp-contract=off" if a.build == "native"
                                else "-O3 -march=x86-64-v2 -ffp-contract=off"),
                      "sample": f"{a.workload} {a.n}^{ndim} in {a.nb}^{ndim} blocks, {a.steps} steps "
                                f"after {a.warmup} warm-up"}))


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark of the B200 finite-volume update (one JSON line on stdout).

Workload: 3D Kelvin-Helmholtz, gamma 1.4, periodic unit cube, 256^3 cells in
512 meshblocks of 32^3 with 3 ghost cells, WENO-Z + HLLC, RK3, CFL 0.4,
synthetic initial state (seeded shear-layer perturbation).  A step is one full
RK3 time step over the whole mesh (three stage launches + the device dt
controller).  Metric: cell-updates/s = interior cells x steps / time.

``value``: the FP32 bulk path (FP64 energy recovery and sums), every block in
one persistent launch per stage, the stage kernel chosen by the library's
autotuner (``config.stage_kernel``), timed with CUDA events on the solver's
stream.  Beside it: the FP64 stage with one launch per mesh, the plain
per-block FP64 path (one launch per meshblock per stage), the FP64 per-task
path (the reference task list, one kernel per task) and the FP32-vs-FP64
density L1.  ``e2e``: the same metric through the C ABI with host buffers:
import of the initial conserved state (interior cells, FP64) from pinned host
memory (finalize derives the primitives and fills the ghost zones),
K x kmy_step (each returns dt to the host), export of the final conserved
state.

``roofline``: the stage kernel against HBM (algorithmic bytes per launch over
its CUDA-event time, of the measured copy bandwidth), with its issue-slot and
FP32-pipe fractions from the per-cell counters of its ncu profile
(profiles/stage_counters.txt) at the sampled SM clock.

``--impl reference`` times the reference's CPU path (the C++ restatement in
oracle/, host-tuned build, all host threads) on the same 256^3 workload.

Multi-GPU (torchrun): the path does not shard here, so every rank runs an
independent replica; the time is the max over ranks and ``value`` the sum.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s"


def args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kmy", choices=["kmy", "reference"])
    ap.add_argument("--n", type=int, default=256, help="cells per dimension")
    ap.add_argument("--nb", type=int, default=32, help="meshblock cells per dimension")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tasks", action="store_true", help="skip the per-task FP64 arm")
    ap.add_argument("--serve", type=int, default=120,
                    help="requests in the serving-stream measurement (0: skip; 2000 = full stream)")
    ap.add_argument("--serve-steps", type=int, default=100)
    ap.add_argument("--serve-seq", type=int, default=240,
                    help="requests solved one after another for the batched/sequential ratio "
                         "(the first N of the stream; all of them when N >= --serve)")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the vortex / Orszag-Tang / adaptive-blast measurements")
    ap.add_argument("--only", choices=["fp32", "fp64"], default=None,
                    help="time one precision only (profiling captures); prints its own line")
    ap.add_argument("--kernel", choices=["brick", "slab", "tune"], default=None,
                    help="stage kernel for --only runs (default: the library's choice)")
    return ap.parse_args()


def workload_config(a, n_gpus):
    nb = (a.n // a.nb) ** 3
    return {
        "workload": f"kelvin_helmholtz_3d {a.n}^3 in {nb} blocks of {a.nb}^3, 3 ghosts, "
                    f"WENO-Z + HLLC, RK3, CFL 0.4",
        "cells": a.n ** 3,
        "meshblocks": nb,
        "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single GPU",
        "cache": state_vs_l2(a.n, a.nb),
    }


def state_vs_l2(n: int, nb: int, ghosts: int = 3) -> str:
    """The line's cache note: the conserved state (5 words per interior cell)
    and a stage's working set (it reads two containers and writes a third,
    ghost zones included) against the 126 MB L2."""
    f64, f32 = 40 * n ** 3 / 1e6, 20 * n ** 3 / 1e6
    padded = (n // nb) ** 3 * (nb + 2 * ghosts) ** 3
    w64, w32 = 3 * 40 * padded / 1e6, 3 * 20 * padded / 1e6
    side = "larger" if w32 > 126.0 else "smaller"
    return (f"inputs {side} than L2 ({n}^3 state: {f64:.0f} MB FP64, {f32:.0f} MB FP32; a stage's three "
            f"containers with ghost zones: {w64:.0f} MB FP64, {w32:.0f} MB FP32)")


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if num(r[1]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][2]),
                "reasons": sorted(reasons), "samples": len(rows),
                "power_w_max": max((num(r[3]) or 0.0) for r in rows)}


# ---------------------------------------------------------------------------
def dist_init():
    """Rank layout from torchrun's environment; a process group over NCCL (gloo
    where no GPU is visible, as in the CPU tests) when there are several ranks.
    The ranks are independent replicas: the group only carries the barrier
    and the max-over-ranks timing."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


def allreduce_max(x: float, ws: int) -> float:
    """Max over ranks (the job's time is its slowest replica's)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(ws: int, cells: int, steps: int, max_ms: float) -> float:
    """Whole-job cell-updates/s: every replica advances `cells` cells `steps`
    times; the job takes the slowest replica's time."""
    return ws * cells * steps / (max_ms / 1e3)


def barrier(ws: int):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def run_stages(s, nstages: int, tasks: bool):
    for st in range(1, nstages + 1):
        if tasks:
            s.task_stage(st, -1.0)
        else:
            s.rk_stage(st)
    s.end_step()


def time_solver(s, stream, K: int, W: int, ws: int, tasks: bool = False, sampler=None):
    """Warm up W steps, then time exactly K steps with CUDA events on the solver's stream."""
    import torch

    ns = s.info.nstages
    for _ in range(W):
        run_stages(s, ns, tasks)
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    ev = [[(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(ns)] for _ in range(K)]
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    launches0 = s.launch_count
    if sampler:
        sampler.start()
    t0.record(stream)
    for k in range(K):
        for st in range(1, ns + 1):
            ev[k][st - 1][0].record(stream)
            if tasks:
                s.task_stage(st, -1.0)
            else:
                s.rk_stage(st)
            ev[k][st - 1][1].record(stream)
        s.end_step()
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    barrier(ws)
    torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    stage_ms = [a.elapsed_time(b) for row in ev for (a, b) in row]
    clk = s.time
    if not (clk["dt"] > 0.0 and clk["dt"] < 1e300):
        raise RuntimeError(f"solver state became non-finite during the timed steps: {clk}")
    return {"total_ms": total_ms, "stage_ms_avg": sum(stage_ms) / len(stage_ms),
            "launches": s.launch_count - launches0, "clocks": clocks}


def make_solver(a, precision: str, device: int, stream, **opts):
    """The workload's solver; opts are <kamayan_b200> deck options
    (stage_kernel, slab_rows, launch)."""
    import kamayan_b200
    from kamayan_b200 import configs

    d = configs.kh_3d(n=a.n, nb=a.nb, precision=precision)
    for k, v in opts.items():
        d.set("kamayan_b200", k, v)
    s = kamayan_b200.Solver(d, device=device)
    s.set_stream(stream.cuda_stream)
    s.pgen("kelvin_helmholtz")
    return s


def e2e_solve(a, device: int, stream, K: int):
    """Initial state from pinned host memory -> K x kmy_step -> final state to pinned host.

    The conserved state moves as interior cells (kmy_import_interior /
    kmy_export_interior, the layout of Parthenon's phdf outputs); finalize
    derives the primitives and fills the ghost zones on the device."""
    import torch

    import kamayan_b200

    src = make_solver(a, "fp64", device, stream)
    names = [("dens", 0), ("momentum", 0), ("momentum", 1), ("momentum", 2), ("ener", 0)]
    n = 1
    for x in src.interior_shape:
        n *= x
    host_in = {}
    for v, c in names:
        t = torch.empty(n, dtype=torch.float64, pin_memory=True)
        src.export_interior_ptr(v, t.data_ptr(), n, c)
        host_in[(v, c)] = t
    src.close()
    host_out = {k: torch.empty(n, dtype=torch.float64, pin_memory=True) for k in names}
    from kamayan_b200 import configs

    s = kamayan_b200.Solver(configs.kh_3d(n=a.n, nb=a.nb, precision="fp32"), device=device)
    s.set_stream(stream.cuda_stream)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for (v, c), t in host_in.items():
        s.import_interior_ptr(v, t.data_ptr(), n, c)
    s.finalize_import()
    for _ in range(K):
        s.step()
    for (v, c), t in host_out.items():
        s.export_interior_ptr(v, t.data_ptr(), n, c)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    s.close()
    h2d = 8 * n * len(names)
    d2h = 8 * n * len(names) + 48 * K
    return ms, h2d, d2h


def stage_counters(kernel: str):
    """Per-cell counters of a stage kernel from its committed ncu summary
    (profiles/stage_counters.txt): DRAM bytes, warp instructions issued, and
    FMA- and XU-pipe busy SM-cycles, per interior cell and stage launch."""
    p = ROOT / "profiles" / "stage_counters.txt"
    try:
        k = json.loads(p.read_text())["kernels"]
        return k.get(kernel) or k.get(kernel + "_fp32")
    except Exception:
        return None


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def cpu_baseline(sample_n: int, min_seconds: float, max_steps: int, steps: int = 1,
                 workload: str = "kh_3d", nb: int = 32, warmup: int = 1, threads: int = 0):
    cmd = [sys.executable, "-m", "oracle.cpu_bench", "--workload", workload, "--n", str(sample_n),
           "--nb", str(nb), "--steps", str(steps), "--warmup", str(warmup), "--min-seconds", str(min_seconds),
           "--max-steps", str(max_steps), "--threads", str(threads), "--build", "native"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=900)
    if r.returncode != 0:
        return {"error": r.stderr[-400:]}
    return json.loads(r.stdout.strip().splitlines()[-1])


def serving_block(a, device: int) -> dict:
    """Serving stream: saturation capacity, Poisson arrivals at 0.8 x capacity,
    and the same requests solved one after another without batching."""
    from kamayan_b200 import serving

    reqs = [serving.make_request(i) for i in range(a.serve)]
    sat = serving.run_stream(reqs, a.serve_steps, arrivals=None, device=device)
    mean_work = sum(r.cells for r in reqs) * a.serve_steps / len(reqs)
    rate = 0.8 * sat["cell_updates_per_s"] / mean_work
    arrivals = serving.poisson_arrivals(len(reqs), rate, seed=11)
    poi = serving.run_stream(reqs, a.serve_steps, arrivals=arrivals, device=device)
    # the same requests, one after another, each on its own context (no batching)
    nseq = min(len(reqs), a.serve_seq)
    seq = serving.run_sequential(reqs[:nseq], a.serve_steps, device=device)
    return {
        "workload": f"{a.serve} requests (seeded mix of vortex/blast, 64^2..128^3, PLM/HLL, PPM/HLLC, "
                    f"WENO-Z/HLLC, FP32/FP64), {a.serve_steps} RK2 steps each",
        "saturation": sat,
        "poisson": dict(poi, offered_load=0.8, rate_per_s=rate),
        "sequential_per_solve": seq,
        "batched_over_sequential": sat["cell_updates_per_s"] / seq["cell_updates_per_s"],
    }


def _evolve_run(s, stream, tlim: float = 1e30, nlim: int = -1):
    """kmy_evolve to tlim (or nlim steps) in one call; device time between two
    events on the solver's stream, the zone-cycles the library counted (each
    step's interior cells on the mesh it ran on, so block-count changes under
    AMR are included) and the steps taken."""
    import torch

    n0, z0 = s.time["ncycle"], s.zone_cycles
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    s.evolve(tlim, nlim)
    t1.record(stream)
    torch.cuda.synchronize()
    return t0.elapsed_time(t1), s.zone_cycles - z0, s.time["ncycle"] - n0


def workloads_block(a, device: int, stream) -> dict:
    """The other configurations of the path on one GPU: 2D vortex to t=10 (FP64,
    fused, kmy_evolve), 3D Orszag-Tang with constrained transport
    (FP32 bulk; fused stage, and the per-task path beside it), and the 2D blast
    on an adaptive mesh to t=0.2."""
    import kamayan_b200
    from kamayan_b200 import configs

    out = {}

    def solver(deck, problem, path):
        s = kamayan_b200.Solver(deck, device=device)
        s.set_stream(stream.cuda_stream)
        s.set_path(path)
        s.pgen(problem)
        return s

    # c1: vortex 128^2, 4 blocks of 64^2, PLM(MC)+HLL, RK2, to t = 10, through
    # kmy_evolve (chunks of steps replayed as CUDA graphs)
    s = solver(configs.vortex_2d(), "isentropic_vortex", "fused")
    ms, upd, steps = _evolve_run(s, stream, tlim=10.0)
    out["vortex_2d_fp64"] = {"cell_updates_per_s": upd / (ms / 1e3), "steps": steps, "seconds": ms / 1e3,
                             "l1_density_vs_exact": s.vortex_error("dens"),
                             "config": "128^2 in 4x64^2, g=2, PLM(MC)+HLL, RK2, CFL 0.8, t=10"}
    s.close()
    # c3: Orszag-Tang 192^3, 216 blocks of 32^3, CT, PPM+HLL, RK2, FP32 bulk;
    # the fused stage (cells) + EMF / face-update kernels, and the per-task path
    n3 = min(a.n, 192)
    ot = {}
    for path in ("fused", "tasks"):
        s = solver(configs.ot_3d(n=n3, nb=32, precision="fp32"), "orszag_tang", path)
        _evolve_run(s, stream, nlim=2)
        ms, upd, steps = _evolve_run(s, stream, nlim=max(3, a.steps // 4))
        ot[path] = (upd / (ms / 1e3), steps, ms / steps, float(abs(s.interior(s.export("divb"))).max()))
        s.close()
    # the same solve to t = 0.5 (the configuration's end time) in FP32 and in
    # FP64: the FP32 run's L1 against FP64 and its div B at t_end
    t_end = {}
    for prec in ("fp32", "fp64"):
        s = solver(configs.ot_3d(n=n3, nb=32, precision=prec), "orszag_tang", "fused")
        ms, upd, steps = _evolve_run(s, stream, tlim=0.5)
        t_end[prec] = (upd / (ms / 1e3), steps, ms / 1e3, s.time["time"],
                       {v: s.interior(s.export(v, c)) for v, c in (("dens", 0), ("ener", 0), ("magc", 0))},
                       float(abs(s.interior(s.export("divb"))).max()))
        s.close()
    l1_ot = {v: float(abs(t_end["fp32"][4][v] - t_end["fp64"][4][v]).sum() / abs(t_end["fp64"][4][v]).sum())
             for v in t_end["fp64"][4]}
    out["orszag_tang_3d_ct_fp32"] = {
        "cell_updates_per_s": ot["fused"][0], "steps": ot["fused"][1], "ms_per_step": ot["fused"][2],
        "max_abs_divb": ot["fused"][3],
        "tasks_cell_updates_per_s": ot["tasks"][0], "tasks_ms_per_step": ot["tasks"][2],
        "to_t_end": {"t_end": t_end["fp32"][3], "steps": t_end["fp32"][1], "seconds_fp32": t_end["fp32"][2],
                     "cell_updates_per_s_fp32": t_end["fp32"][0], "seconds_fp64": t_end["fp64"][2],
                     "cell_updates_per_s_fp64": t_end["fp64"][0], "l1_fp32_vs_fp64": l1_ot,
                     "max_abs_divb_fp32": t_end["fp32"][5], "max_abs_divb_fp64": t_end["fp64"][5]},
        "config": f"{n3}^3 in 32^3 blocks, g=4, CT, PPM(MC)+HLL, RK2, CFL 0.3, fused stage"}
    # c4: blast on an adaptive mesh, 128^2 base in 16^2 blocks, 3 levels,
    # Loehner on density, to t = 0.2, in FP64 and FP32
    amr = {}
    for prec in ("fp64", "fp32"):
        s = solver(configs.blast_2d_amr(precision=prec), "blast", "tasks")
        nb0 = s.nblocks
        ms, upd, steps = _evolve_run(s, stream, tlim=0.2)
        # the steps' device time as kmy_evolve counted it (host read-backs and
        # tree updates excluded): the wall-over-device ratio is the host's share
        dev = s.evolve_device_ms
        amr[prec] = {"cell_updates_per_s": upd / (ms / 1e3), "steps": steps, "seconds": ms / 1e3,
                     "device_seconds": dev / 1e3, "wall_over_device": ms / dev if dev > 0 else None,
                     "blocks_initial": nb0, "blocks_final": s.nblocks, "leaves": s.blocks(),
                     "dens": s.interior(s.export("dens"))}
        s.close()
    a64, a32 = amr["fp64"], amr["fp32"]
    same = (a64["leaves"][0].shape == a32["leaves"][0].shape and bool((a64["leaves"][0] == a32["leaves"][0]).all())
            and bool((a64["leaves"][1] == a32["leaves"][1]).all()))
    out["blast_2d_amr_fp64"] = {k: v for k, v in a64.items() if k not in ("leaves", "dens")}
    out["blast_2d_amr_fp64"]["config"] = \
        "128^2 base in 16^2 blocks, 3 levels, Loehner dens 0.3/0.05, PLM(MC)+HLLC, RK2, t=0.2"
    out["blast_2d_amr_fp64"]["fp32"] = {
        "cell_updates_per_s": a32["cell_updates_per_s"], "steps": a32["steps"], "blocks_final": a32["blocks_final"],
        "wall_over_device": a32["wall_over_device"],
        "same_leaves_as_fp64": same,
        "l1_density_vs_fp64": (float(abs(a32["dens"] - a64["dens"]).sum() / abs(a64["dens"]).sum())
                               if same else None)}
    return out


def main_reference(a):
    # the reference's CPU path runs once, on rank 0; other ranks have no work
    # and need no process group
    if int(os.environ.get("RANK", "0")) != 0:
        return
    # the full workload (256^3 in 512 blocks of 32^3), all host threads,
    # host-tuned build; a step takes a few seconds, so K is bounded
    steps = max(1, min(a.steps, 3))
    cb = cpu_baseline(a.n, 0.0, steps, steps=steps, nb=a.nb, warmup=1)
    cfg = workload_config(a, a.gpus)
    line = {
        "impl": "reference", "metric": METRIC, "value": cb.get("value"), "unit": METRIC,
        "n_gpus": a.gpus, "steps": cb.get("steps"), "warmup": 1, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": cb.get("value"), "unit": METRIC, "cores": cb.get("threads"),
                         "kind": "port", "sample": cb.get("sample"), "cpu": cb.get("cpu"),
                         "build": cb.get("build")},
        "e2e": {"value": cb.get("value"), "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference's own build is unavailable (un-vendored Parthenon/Kokkos); "
                "timed: the C++ restatement of its CPU path, OpenMP over meshblocks, on the same workload",
    }
    print(json.dumps(line), flush=True)


def main():
    a = args()
    if a.impl == "reference":
        return main_reference(a)
    import torch

    ws, rank, local = dist_init()
    device = local
    torch.cuda.set_device(device)
    stream = torch.cuda.Stream(device=device)
    K, W = a.steps, max(3, a.warmup)
    cells = a.n ** 3
    ns = 3

    if a.only:
        s1 = make_solver(a, a.only, device, stream, **({"stage_kernel": a.kernel} if a.kernel else {}))
        r1 = time_solver(s1, stream, K, W, ws)
        kern = s1.stage_kernel
        s1.close()
        tot = allreduce_max(r1["total_ms"], ws)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": job_value(ws, cells, K, tot), "unit": METRIC,
                              "n_gpus": ws, "steps": K, "warmup": W, "ms_per_step": tot / K,
                              "dtype": "f32" if a.only == "fp32" else "f64", "stage_kernel": kern,
                              "launch_ms_avg": r1["stage_ms_avg"], "config": workload_config(a, ws),
                              "note": f"{a.only}-only profiling run; not the headline line"}),
                  flush=True)
        return

    # headline: FP32 bulk path, the stage kernel the autotuner picks for this
    # device and configuration (timed on the solver's state before the warm-up)
    s32 = make_solver(a, "fp32", device, stream, stage_kernel="tune")
    tuning = s32.autotune(reps=3)
    kernel = s32.stage_kernel
    sampler = ClockSampler(device)
    r32 = time_solver(s32, stream, K, W, ws, sampler=sampler)
    # FP64, one launch per stage over the whole mesh
    s64 = make_solver(a, "fp64", device, stream)
    r64 = time_solver(s64, stream, K, W, ws)
    import numpy as np

    d32 = s32.interior(s32.export("dens"))
    d64 = s64.interior(s64.export("dens"))
    l1 = float(np.abs(d32 - d64).sum() / np.abs(d64).sum())
    t32, t64 = s32.time["time"], s64.time["time"]
    s32.close()
    s64.close()
    # the plain per-block FP64 path: the same stage kernel, one launch per
    # meshblock per stage
    Kp = max(2, K // 4)
    spb = make_solver(a, "fp64", device, stream, launch="per_block")
    rpb = time_solver(spb, stream, Kp, W, ws)
    spb.close()
    # FP64 per-task path (the reference task list as separate kernels)
    rt = None
    if not a.no_tasks:
        st = make_solver(a, "fp64", device, stream)
        st.set_path("tasks")
        rt = time_solver(st, stream, max(2, K // 4), W, ws, tasks=True)
        st.close()
    e2e_ms, h2d, d2h = e2e_solve(a, device, stream, K)

    tot32 = allreduce_max(r32["total_ms"], ws)
    tot64 = allreduce_max(r64["total_ms"], ws)
    totpb = allreduce_max(rpb["total_ms"], ws)
    e2e_ms = allreduce_max(e2e_ms, ws)
    value = job_value(ws, cells, K, tot32)
    v64 = job_value(ws, cells, K, tot64)
    vpb = job_value(ws, cells, Kp, totpb)
    vt = None
    if rt:
        Kt = max(2, K // 4)
        vt = ws * cells * Kt / (allreduce_max(rt["total_ms"], ws) / 1e3)

    # roofline of the dominant kernel (the stage): algorithmic bytes per
    # launch = cells x words x bytes, words = 10 (stage 1) or 15 (stages 2, 3)
    # (5 conserved words per cell; the FP32 path's energy low word not counted)
    words_avg = (10 + 15 * (ns - 1)) / ns
    alg32 = cells * words_avg * 4
    alg64 = cells * words_avg * 8
    peak, peak_kind = peaks()
    launch_s = r32["stage_ms_avg"] / 1e3
    ach32 = alg32 / launch_s / 1e9
    ach64 = alg64 / (r64["stage_ms_avg"] / 1e3) / 1e9
    ctr = stage_counters(kernel)
    clk = r32["clocks"] or {}
    mhz = clk.get("sm_mhz") or clk.get("sm_max_mhz") or 1965.0
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    roof = {"bound": "hbm", "achieved": ach32, "peak": peak, "unit": "GB/s", "frac": ach32 / peak,
            "traffic": (ctr["dram_bytes_per_cell"] * cells) if ctr else None, "peak_kind": peak_kind,
            "kernel": kernel, "alg_bytes_per_launch": alg32, "launch_ms_avg": r32["stage_ms_avg"]}
    if ctr:
        cyc = launch_s * mhz * 1e6 * sms  # SM-cycles of one launch
        roof["issue"] = {"frac": ctr["warp_inst_per_cell"] * cells / (cyc * 4),
                         "what": "warp instructions issued / (4 schedulers x SMs x cycles of the launch)"}
        if "fma_pipe_sm_cycles_per_cell" in ctr:
            roof["fp32_pipe"] = {"frac": ctr["fma_pipe_sm_cycles_per_cell"] * cells / cyc,
                                 "xu_frac": ctr["xu_pipe_sm_cycles_per_cell"] * cells / cyc,
                                 "what": "FMA-pipe (and reciprocal/XU-pipe) busy SM-cycles / SM-cycles of the launch"}
        roof["counters"] = f"profiles/stage_counters.txt ({ctr.get('source', '')})"

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": tot32 / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "config": dict(workload_config(a, ws), stage_kernel=kernel),
        "e2e": {"value": job_value(ws, cells, K, e2e_ms), "unit": METRIC,
                "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
                "what": "kmy_import_interior of the conserved state (FP64 interior cells, pinned host) + "
                        "finalize + K x kmy_step + kmy_export_interior of the conserved state, FP32 solve"},
        "gpu_launches": r32["launches"],
        "roofline": roof,
        "clocks": r32["clocks"],
        "tuning": {k: v for k, v in tuning.items()},
        "fp64_fused": {"value": v64, "ms_per_step": tot64 / K, "launch_ms_avg": r64["stage_ms_avg"],
                       "roofline_achieved_gbs": ach64, "frac": ach64 / peak},
        "fp64_per_block": {"value": vpb, "ms_per_step": totpb / Kp, "steps": Kp,
                           "what": "the FP64 brick stage launched once per meshblock per stage"},
        "fp64_tasks": ({"value": vt, "ms_per_step": rt["total_ms"] / max(2, K // 4)} if rt else None),
        "fp32_over_fp64_per_block": value / vpb,
        "fp32_over_fp64_fused": value / v64,
        "l1_density_fp32_vs_fp64": l1,
        "sim_time_fp32_fp64": [t32, t64],
    }
    if not a.no_workloads:
        line["workloads"] = wl = workloads_block(a, device, stream)
        if rank == 0 and ws == 1 and not a.no_cpu_baseline:
            # the oracle on bounded samples of the same workloads (all host threads)
            for key, args_ in (("vortex_2d_fp64", dict(workload="vortex_2d", sample_n=128, nb=64, steps=200)),
                               ("orszag_tang_3d_ct_fp32", dict(workload="ot_3d", sample_n=64, nb=32, steps=1)),
                               ("blast_2d_amr_fp64", dict(workload="blast_2d_amr", sample_n=128, nb=16,
                                                          steps=100, warmup=0))):
                cb = cpu_baseline(min_seconds=0.0, max_steps=args_["steps"], **args_)
                wl[key]["cpu_sample"] = {"value": cb.get("value"), "cores": cb.get("threads"),
                                         "sample": cb.get("sample"), "kind": "port"}
    if a.serve > 0:
        line["serving"] = serving_block(a, device)
    if rank == 0 and ws == 1 and not a.no_cpu_baseline:
        # the same 256^3 workload on all host threads (one step after one
        # warm-up step), and on one core a 128^3 sample of it
        cb = cpu_baseline(a.n, 0.0, 1, steps=1, nb=a.nb, warmup=1)
        c1 = cpu_baseline(128, 0.0, 1, steps=1, nb=a.nb, warmup=0, threads=1)
        line["cpu_baseline"] = {"value": cb.get("value"), "unit": METRIC, "cores": cb.get("threads"),
                                "kind": "port", "sample": cb.get("sample"), "cpu": cb.get("cpu"),
                                "build": cb.get("build"),
                                "one_core": {"value": c1.get("value"), "sample": c1.get("sample")}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()

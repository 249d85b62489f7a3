"""The multi-GPU arrangement of bench.py on CPU: two gloo ranks (127.0.0.1).

The path does not shard (each GPU runs an independent replica), so the only
cross-rank steps are the barrier before the timed region and the max over
ranks of the measured time; the job's value is the replicas' summed work over
the slowest replica's time.  This checks those steps with world size 2, and
that the reference arm does its work on rank 0 alone.
"""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

CHILD = r'''
import os, sys, json
sys.path.insert(0, sys.argv[1])
import bench
ws, rank, local = bench.dist_init()
import torch.distributed as dist
assert dist.get_backend() == "gloo" and ws == 2 and local == rank
bench.barrier(ws)
# rank r measured 10 + 5 r ms; the job time is the slower rank's
t = bench.allreduce_max(10.0 + 5.0 * rank, ws)
v = bench.job_value(ws, 1000, 4, t)
print(json.dumps({"rank": rank, "t": t, "v": v}), flush=True)
bench.barrier(ws)
dist.destroy_process_group()
'''


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(code: str, args: list[str], ws: int = 2, extra_env: dict | None = None):
    port = _free_port()
    procs = []
    for r in range(ws):
        env = dict(os.environ, WORLD_SIZE=str(ws), RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        env.update(extra_env or {})
        procs.append(subprocess.Popen([sys.executable, "-c", code, *args], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        o, e = p.communicate(timeout=180)
        assert p.returncode == 0, e[-2000:]
        out.append(o)
    return out


def test_two_ranks_take_the_slower_time():
    import json

    outs = _launch(CHILD, [str(ROOT)])
    res = [json.loads([ln for ln in o.splitlines() if ln.startswith("{")][-1]) for o in outs]
    for r in res:
        assert r["t"] == 15.0
        # two replicas of 1000 cells x 4 steps in 15 ms
        assert r["v"] == pytest.approx(2 * 1000 * 4 / 0.015)


def test_reference_arm_runs_on_rank_zero_only():
    # rank 1 of a two-rank reference launch exits at once without output
    code = "import sys; sys.path.insert(0, sys.argv[1]); sys.argv = ['bench.py', '--impl', 'reference']; " \
           "import bench; bench.main_reference(bench.args())"
    port = _free_port()
    env = dict(os.environ, WORLD_SIZE="2", RANK="1", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([sys.executable, "-c", code, str(ROOT)], env=env, capture_output=True, text=True,
                       timeout=120)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""

"""The multi-GPU plumbing of bench.py on the CPU: two ranks over gloo (the GPU
runs use NCCL the same way).  Instances are replicas, so the only collectives
are the barrier and the max of the per-rank times; the whole-job value is
world x steps / slowest rank's time.  The reference arm runs on rank 0 only."""
import json
import os
import socket
import subprocess
import sys

from conftest import ROOT

WORKER = r"""
import json, os, sys
sys.path.insert(0, os.getcwd())
import bench
r = bench.Ranks("gloo", timeout_s=60)
r.barrier()
ms = 100.0 * (r.rank + 1)          # rank 1 is the slow one
m = r.gmax(ms)
print(json.dumps({"rank": r.rank, "world": r.world, "max_ms": m, "value": bench.replica_value(r.world, 3, m)}))
r.close()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _env(rank, world, port):
    e = dict(os.environ)
    e.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
             MASTER_PORT=str(port))
    return e


def test_two_gloo_ranks_take_the_max_time_and_sum_the_replicas():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", WORKER], cwd=ROOT, env=_env(r, 2, port),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["world"] == 2
        assert o["max_ms"] == 200.0
        assert abs(o["value"] - 2 * 3 / 0.2) < 1e-9
    assert sorted(o["rank"] for o in outs) == [0, 1]


def test_reference_arm_runs_on_rank_zero_only():
    args = ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0",
            "--n", "64", "--nt", "40", "--cpu-steps", "4"]
    r1 = subprocess.run([sys.executable] + args, cwd=ROOT, env=_env(1, 2, _free_port()), capture_output=True,
                        text=True, timeout=300)
    assert r1.returncode == 0 and r1.stdout.strip() == ""
    r0 = subprocess.run([sys.executable] + args, cwd=ROOT, env=_env(0, 2, _free_port()), capture_output=True,
                        text=True, timeout=300)
    assert r0.returncode == 0, r0.stderr[-2000:]
    line = json.loads(r0.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0

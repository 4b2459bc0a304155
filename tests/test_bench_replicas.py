"""The N > 1 path of bench.py on the CPU: two gloo ranks launched as
torchrun would (RANK / WORLD_SIZE / MASTER_* in the environment) run
independent replicas; the whole-job rate uses the slowest rank's time, and
the reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import os, sys, datetime
sys.path.insert(0, {root!r})
import torch, torch.distributed as dist
import bench
rank, world, local = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
t_local = 1.0 + rank          # rank 1 is the slower replica
rate, t_max = bench.replica_rate(torch, 100, t_local, world, "cpu")
print("RESULT", rank, world, rate, t_max, flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(code, world=2, extra=None):
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code] + (extra or []), env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True))
    outs = []
    for p in procs:
        try:
            out, _ = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            out, _ = p.communicate()
        outs.append((p.returncode, out))
    return outs


def test_replica_rate_uses_the_slowest_rank():
    outs = run_ranks(CHILD.format(root=ROOT))
    res = {}
    for rc, out in outs:
        assert rc == 0, out
        line = [l for l in out.splitlines() if l.startswith("RESULT")][0].split()
        res[int(line[1])] = (int(line[2]), float(line[3]), float(line[4]))
    for r in (0, 1):
        world, rate, t_max = res[r]
        assert world == 2
        assert t_max == pytest.approx(2.0)          # max over ranks
        assert rate == pytest.approx(2 * 100 / 2.0)  # all ranks' steps over that time


def test_reference_arm_non_zero_rank_exits_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""

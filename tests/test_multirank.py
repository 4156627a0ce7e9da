"""The multi-GPU host logic on the CPU: two gloo ranks.

bench.py runs one replica per GPU (each rank renders its own frame; no data
exchange): the whole-job value is every rank's rays over the slowest rank's
device time, and only rank 0 prints; the reference arm runs on rank 0 alone.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import json, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
dist.init_process_group("gloo")
rank = dist.get_rank()
ms, rays = bench.combine_over_ranks(100.0 + 50.0 * rank, 1000.0 * (rank + 1), dist, "cpu")
print(json.dumps({"rank": rank, "ms": ms, "rays": rays}), flush=True)
dist.barrier()
dist.destroy_process_group()
'''


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_slowest_time_and_every_rays():
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE="2",
                   LOCAL_RANK=str(rank))
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["ms"] == 150.0  # the slower rank's time
        assert o["rays"] == 3000.0  # both ranks' rays


def test_one_rank_keeps_its_own_figures():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.combine_over_ranks(12.5, 7, None, "cpu") == (12.5, 7.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import bench

    class Args:
        pass

    assert bench.run_reference(Args(), 1) is None  # rank 1 returns before any work
    assert capsys.readouterr().out == ""

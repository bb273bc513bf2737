"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1) combine their
device times as the maximum over ranks and report whole-job throughput; the reference arm
prints from rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import os, sys, json
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
rank, ws = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="env://")
# rank r is slower on the first value, faster on the second
t = bench.slowest([10.0 + 5.0 * rank, 7.0 - 3.0 * rank], ws, "cpu")
rate = bench.job_rate(1000.0, ws, t[0])
print(json.dumps({"rank": rank, "t": t, "rate": rate}))
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_gloo_ranks_take_max_time():
    port = _free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE="2", LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["t"] == [15.0, 7.0]
        assert o["rate"] == pytest.approx(2 * 1000.0 / 0.015)


def test_reference_arm_prints_from_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        scene, steps, warmup, gpus = "config1", 1, 1, 2
    assert bench.run_reference(A) == 0
    assert capsys.readouterr().out == ""

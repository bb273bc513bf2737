"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (127.0.0.1) combine their
device times as the maximum over ranks and report whole-job throughput, split the batched
block's scenes between them and join their shares after the timed region; the reference
arm prints from rank 0 only."""
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


SHARD_WORKER = r"""
import os, sys, json
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
from snowsimulation_b200.batch import shard_scenes
rank, ws = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="env://")
sizes = [100 + 37 * k for k in range(10)]
mine = shard_scenes(sizes, ws, rank)
frames = 2
# what batched_compare returns, with device times made up (rank 1 the slower one)
part = {"frames": frames, "scenes_total": len(sizes), "particles_total": sum(sizes), "boundary_total": 7,
        "scenes": mine, "particle_substeps": sum(sizes[i] for i in mine) * bench.SUBSTEPS * frames,
        "batch_ms": 10.0 + 2.0 * rank, "plain_ms": 30.0 - 4.0 * rank,
        "water_after": [i for i in mine], "snow_after": [sizes[i] - i for i in mine]}
parts = [None] * ws
dist.all_gather_object(parts, part)
print(json.dumps({"rank": rank, "line": bench.combine_batched(parts)}))
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


def _run_ranks(worker, n=2):
    port = _free_port()
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(n), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", worker, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    return outs


def test_two_gloo_ranks_split_the_batched_scenes():
    outs = _run_ranks(SHARD_WORKER)
    sizes = [100 + 37 * k for k in range(10)]
    total = sum(sizes)
    for o in outs:
        line = o["line"]
        assert line == outs[0]["line"]   # every rank holds the same joined figures
        assert sum(line["scenes_per_rank"]) == 10
        assert sum(line["particles_per_rank"]) == total
        # all scenes' particle-substeps over the slowest rank's batch (12 ms) and plain (30 ms) time
        ps = total * 4 * 2
        assert line["value"] == pytest.approx(ps / 0.012)
        assert line["plain_value"] == pytest.approx(ps / 0.030)
        assert line["ms_per_step"] == pytest.approx(6.0)
        assert line["parallelism"] == "scenes split over 2 ranks"
        assert line["particles_after"] == {"water": sum(range(10)), "snow": total - sum(range(10))}


def test_combine_batched_rejects_a_lost_or_doubled_scene():
    sys.path.insert(0, ROOT)
    import bench

    def part(scenes):
        return {"frames": 1, "scenes_total": 3, "particles_total": 30, "boundary_total": 0, "scenes": scenes,
                "particle_substeps": 40 * len(scenes), "batch_ms": 1.0, "plain_ms": 2.0,
                "water_after": [0] * len(scenes), "snow_after": [10] * len(scenes)}
    assert bench.combine_batched([part([0, 2]), part([1])])["scenes_per_rank"] == [2, 1]
    with pytest.raises(RuntimeError):
        bench.combine_batched([part([0, 1]), part([1, 2])])
    with pytest.raises(RuntimeError):
        bench.combine_batched([part([0]), part([2])])


def test_reference_arm_prints_from_rank0_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        scene, steps, warmup, gpus = "config1", 1, 1, 2
    assert bench.run_reference(A) == 0
    assert capsys.readouterr().out == ""

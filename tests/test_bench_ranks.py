"""The bench's multi-rank host logic on CPU ranks (gloo, world size 2): the
job's timings are the maximum over ranks, every rank gets the same values,
and the reference arm runs on rank 0 only (the other ranks exit 0 silently)."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

RANK_SCRIPT = """
import datetime, json, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
out = bench.max_over_ranks([1.0 + rank, 10.0 - 3 * rank, 2.5], "cpu", world)
single = bench.max_over_ranks([1.0 + rank], "cpu", 1)       # one rank: no collective
dist.barrier()
dist.destroy_process_group()
print(json.dumps({"rank": rank, "out": out, "single": single}))
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env(rank, world, port):
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
               WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    env.pop("CUDA_VISIBLE_DEVICES", None)
    return env


def test_max_over_ranks_two_gloo_ranks():
    port = _free_port()
    procs = [subprocess.Popen([sys.executable, "-c", RANK_SCRIPT, str(ROOT)], env=_env(r, 2, port),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for r in range(2)]
    outs = []
    for p in procs:
        try:
            o, e = p.communicate(timeout=180)
        finally:
            if p.poll() is None:
                p.kill()
        assert p.returncode == 0, e[-2000:]
        outs.append(json.loads(o.strip().splitlines()[-1]))
    for d in outs:
        assert d["out"] == [2.0, 10.0, 2.5]
        assert d["single"] == [1.0 + d["rank"]]


def test_reference_arm_other_ranks_exit_silently():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=_env(1, 2, _free_port()), cwd=str(ROOT),
                       capture_output=True, text=True, timeout=180)
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""
